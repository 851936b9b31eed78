"""Sampled runs: the device sampler, the start-state geometry, the CCS
reduction and its determinism."""
import numpy as np
import pytest

from cosims_b200 import abi, engine
from oracle import oracle
from tests.common import load

pytestmark = pytest.mark.gpu


def test_start_states_match_oracle_geometry():
    """Device start states from the sampled (b, phi, theta, gamma, g) agree with
    the oracle's restatement of monteTraj.cpp:235-269 to rounding (the device
    uses CUDA's sin/cos)."""
    mol, par, _ = load("q128_t1")
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        ins, pos0, vel0, hit = ctx.sample_inputs(seed=5, first=1000, n=5000)
    p1, v1, h1 = oracle.start_states(par, ins)
    agree = hit == h1
    assert agree.mean() > 0.999            # a grazing ray can flip on rounding
    sel = agree & (hit == 1)
    np.testing.assert_allclose(pos0[sel], p1[sel], rtol=0, atol=1e-10)
    np.testing.assert_allclose(vel0[sel], v1[sel], rtol=1e-14, atol=1e-12)


def test_sampler_distributions():
    """theta ~ sin(theta), b ~ b on [0, b_max], g within [g_min, g_max]
    following g^5 exp(-a g^2) (monteTraj.cpp:203-231)."""
    mol, par, _ = load("c1_t3")
    with engine.Context(mol, par, abi.MIXED) as ctx:
        ins, _, _, _ = ctx.sample_inputs(seed=3, first=0, n=200000)
    b = ins["b"] / par.b_max
    assert abs(np.mean(b) - 2 / 3) < 0.005           # E[b] = 2/3 b_max
    assert abs(np.mean(np.cos(ins["theta"]))) < 0.01  # uniform cos(theta)
    assert abs(np.mean(ins["phi"]) - np.pi) < 0.02
    g = ins["g"]
    assert g.min() >= par.g_min and g.max() <= par.g_max
    grid = np.linspace(par.g_min, par.g_max, 4001)
    pdf = grid ** 5 * np.exp(-par.vdist_a * grid ** 2)
    mean = np.sum(grid * pdf) / np.sum(pdf)
    assert abs(np.mean(g) - mean) / mean < 0.005


def test_sampled_run_matches_oracle_on_same_inputs():
    """A sampled plain run = the oracle run on the device's sampled inputs,
    with the reference's CCS bookkeeping (n_eff) reproduced exactly."""
    mol, par, _ = load("q128_t1")
    n = 1500
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        s, ins, outs = ctx.run_sampled(seed=17, first=0, n=n, update_every=400,
                                       want_records=True)
        ins2, pos0, vel0, hit = ctx.sample_inputs(seed=17, first=0, n=n)
    np.testing.assert_array_equal(ins, ins2)
    assert np.array_equal((outs["status"] & abi.TRAJ_HIT) > 0, hit == 1)
    sel = hit == 1
    ref = oracle.run_list(mol, par, pos0[sel], vel0[sel])
    assert np.max(np.abs(outs["chi"][sel] - ref["chi"])) <= 1e-12
    np.testing.assert_array_equal(outs["status"][sel], ref["status"])
    rs = oracle.reduce(par, outs, 400)
    assert s.n == n and s.n_hit == rs.n_hit and s.n_success == rs.n_success
    assert s.n_eff == rs.n_eff
    assert abs(s.sum - rs.sum) <= 1e-9 * abs(rs.sum)
    assert abs(s.sum2 - rs.sum2) <= 1e-9 * abs(rs.sum2)
    assert s.steps >= int(outs["steps"].sum())
    assert s.force_evals > s.steps and s.pair_es + s.pair_lj > 0


@pytest.mark.parametrize("precision", [abi.PLAIN_F64, abi.MIXED])
def test_sampled_sums_deterministic_across_launch_shapes(precision):
    mol, par, _ = load("c0_t5")
    with engine.Context(mol, par, precision) as ctx:
        s1, _, o1 = ctx.run_sampled(seed=9, first=0, n=3000, update_every=1000, want_records=True)
        ctx.set_launch(block_threads=64)
        s2, _, o2 = ctx.run_sampled(seed=9, first=0, n=3000, update_every=1000, want_records=True)
    np.testing.assert_array_equal(o1, o2)
    assert s1.sum == s2.sum and s1.sum2 == s2.sum2 and s1.n_eff == s2.n_eff


def test_run_is_independent_of_batching():
    """Trajectory i of a stream depends only on (seed, i): one run of 2000
    equals runs of 700 + 1300 with the matching first index."""
    mol, par, _ = load("c0_t5")
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        _, _, a = ctx.run_sampled(seed=21, first=0, n=2000, want_records=True)
        _, _, b1 = ctx.run_sampled(seed=21, first=0, n=700, want_records=True)
        _, _, b2 = ctx.run_sampled(seed=21, first=700, n=1300, want_records=True)
    np.testing.assert_array_equal(a, np.concatenate([b1, b2]))


@pytest.mark.parametrize("precision", [abi.PLAIN_F64, abi.MIXED])
@pytest.mark.parametrize("name", ["c0_t5", "c1_t3"])
def test_run_integrals_equals_separate_integrals(name, precision):
    """cosims_run_integrals: integral k of one call is bit for bit a separate
    cosims_run_sampled of trajectories first + k n .. (the same sums and n_eff),
    and the call's work counters are the separate runs' summed."""
    mol, par, _ = load(name)
    n, k, first, every = 3000, 3, 500, 700
    with engine.Context(mol, par, precision) as ctx:
        many, work = ctx.run_integrals(seed=13, first=first, n_per=n, n_integrals=k,
                                       update_every=every)
        sep = [ctx.run_sampled(seed=13, first=first + i * n, n=n, update_every=every)[0]
               for i in range(k)]
    for a, b in zip(many, sep):
        assert (a.sum, a.sum2, a.max_de_pct, a.n, a.n_hit, a.n_success, a.n_eff) == \
            (b.sum, b.sum2, b.max_de_pct, b.n, b.n_hit, b.n_success, b.n_eff)
        assert a.steps == 0 and a.pair_es == 0            # work is reported for the call
    assert work.steps == sum(b.steps for b in sep)
    assert work.force_evals == sum(b.force_evals for b in sep)
    assert work.pair_lj + work.pair_es == sum(b.pair_lj + b.pair_es for b in sep)
    assert work.pair_es_nolj == sum(b.pair_es_nolj for b in sep)
    assert work.sum == 0 and work.n == 0


@pytest.mark.parametrize("precision", [abi.PLAIN_F64, abi.MIXED])
def test_reserve_allocates_before_the_calls(precision):
    """cosims_ctx_reserve: after it, calls within the reserved size take no
    device memory, and their sums equal those of a context that grew its
    buffers in the calls."""
    import torch
    mol, par, _ = load("c0_t5")
    n, k = 2000, 4
    with engine.Context(mol, par, precision) as fresh:
        want, _ = fresh.run_integrals(seed=5, first=0, n_per=n, n_integrals=k)
    with engine.Context(mol, par, precision) as ctx:
        ctx.reserve(n * k, k)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        got, _ = ctx.run_integrals(seed=5, first=0, n_per=n, n_integrals=k)
        ctx.run_sampled(seed=5, first=0, n=n * k)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        with pytest.raises(engine.CosimsError):
            ctx.reserve(-1, 1)
    for a, b in zip(got, want):
        assert (a.sum, a.sum2, a.n_hit, a.n_eff) == (b.sum, b.sum2, b.n_hit, b.n_eff)


@pytest.mark.parametrize("precision", [abi.PLAIN_F64, abi.MIXED])
def test_charge_only_pairs_counted(precision):
    """pair_es_nolj: the charge-field pairs outside the LJ cut-off (variant 3's
    clusters beyond the dispersion radius), a subset of pair_es; none for the
    neutral variant 5.  Both forms count the same clusters, so on the same
    sampled trajectories their shares agree closely."""
    shares = {}
    for name in ("c1_t3", "c0_t5"):
        mol, par, _ = load(name)
        with engine.Context(mol, par, precision) as ctx:
            s, _, _ = ctx.run_sampled(seed=3, first=0, n=2000)
        if name == "c0_t5":
            assert s.pair_es_nolj == 0
        else:
            assert 0 < s.pair_es_nolj < s.pair_es
            shares[name] = s.pair_es_nolj / s.pair_es
    assert 0.2 < shares["c1_t3"] < 0.95
