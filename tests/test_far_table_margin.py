"""The far-field table's FP32 near/far tests (variants 1 and 2 of the mixed
form) against the FP64 tests they stand for.

The kernel forms the He-cluster separation from FP32 hi/lo pairs,
dx = (x_hi - c_hi) + (x_lo - c_lo), squares and sums it in FP32 and compares
the square with the FP32 radii.  Within 2^-16 (relative) of a radius it
repeats the test in FP64 on the cluster record, so every decision is the FP64
test's as long as the FP32 square is within 2^-16 of the FP64 one whenever
the two tests could disagree.  This restates the kernel's arithmetic in numpy
float32 (IEEE round-to-nearest, as the packed FP32 instructions) and checks
that bound and the decisions, on random and on near-threshold separations."""
import numpy as np

MARGIN = np.float32(1.0 / 65536.0)


def _hi_lo(v):
    hi = v.astype(np.float32)
    lo = (v - hi.astype(np.float64)).astype(np.float32)
    return hi, lo


def _fp32_square(pos, ctr):
    """The table pass's squared separation: negated centres as stored, then
    (h + (-c_hi)) + (l + (-c_lo)) per axis, squares, (xx + yy) + zz."""
    h, l = _hi_lo(pos)
    ch, cl = _hi_lo(ctr)
    d = ((h + (-ch)).astype(np.float32) + (l + (-cl)).astype(np.float32)).astype(np.float32)
    sq = (d * d).astype(np.float32)
    return ((sq[:, 0] + sq[:, 1]).astype(np.float32) + sq[:, 2]).astype(np.float32)


def _fp64_square(pos, ctr):
    d = pos - ctr
    return d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]


def test_fp32_square_within_margin_of_fp64():
    rng = np.random.default_rng(17)
    n = 400_000
    pos = rng.uniform(-120.0, 120.0, size=(n, 3))
    ctr = rng.uniform(-60.0, 60.0, size=(n, 3))
    r2f = _fp32_square(pos, ctr).astype(np.float64)
    r2d = _fp64_square(pos, ctr)
    far = r2d > 1.0                      # the radii (r_mp + R)^2 are tens of square Angstrom
    rel = np.abs(r2f[far] - r2d[far]) / r2d[far]
    assert rel.max() < float(MARGIN) / 8


def test_decisions_outside_the_margin_equal_fp64():
    rng = np.random.default_rng(23)
    n = 400_000
    ctr = rng.uniform(-60.0, 60.0, size=(n, 3))
    radius2 = rng.uniform(100.0, 900.0, size=n)          # (12 A + cluster radius)^2 and so on
    # separations placed around the radius, many within a few ulps of it
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    scale = 1.0 + rng.choice([1e-3, 1e-5, 1e-7, 1e-9], size=n) * rng.uniform(-1, 1, size=n)
    pos = ctr + u * (np.sqrt(radius2) * scale)[:, None]
    r2f = _fp32_square(pos, ctr)
    thr = radius2.astype(np.float32)
    r2d = _fp64_square(pos, ctr)
    decided = np.abs(r2f - thr) > MARGIN * thr            # the FP32 test stands
    assert decided.sum() > n // 4 and (~decided).sum() > n // 4
    np.testing.assert_array_equal((r2f > thr)[decided], (r2d > radius2)[decided])


def test_null_entries_are_far_and_never_ambiguous():
    """Null entries carry radii -1: every finite square is beyond them, and
    |r2 - (-1)| <= 2^-16 * (-1) never holds."""
    r2 = np.float32([0.0, 1.0, 3.0e8])
    thr = np.float32(-1.0)
    assert (r2 > thr).all()
    assert not (np.abs(r2 - thr) <= MARGIN * thr).any()
