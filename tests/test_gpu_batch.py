"""Batched form: many molecules in one persistent launch."""
import numpy as np
import pytest

from cosims_b200 import abi, engine
from tests.common import load

pytestmark = pytest.mark.gpu

NAMES = ["c0_t5", "q128_t1", "c1_t3", "q128_t4", "q128_t2"]


def _setup():
    loaded = [load(n) for n in NAMES]
    return [m for m, _, _ in loaded], [p for _, p, _ in loaded]


def test_batch_alone_equals_in_the_mix():
    """A molecule's sums do not depend on the other molecules of the batch."""
    mols, pars = _setup()
    k = len(mols)
    seeds = np.arange(100, 100 + k)
    first = np.zeros(k, np.int64)
    n = np.full(k, 3000)
    with engine.Batch(mols, pars) as b:
        mix = b.run(seeds, first, n)
        for m in range(k):
            only = np.zeros(k, np.int64)
            only[m] = n[m]
            alone = b.run(seeds, first, only)
            a, x = alone[m], mix[m]
            assert (a.sum, a.sum2, a.n, a.n_hit, a.n_eff) == (x.sum, x.sum2, x.n, x.n_hit, x.n_eff)


def test_batch_matches_single_molecule_context():
    """Same sampled inputs as the single-molecule mixed path (same lanes per
    trajectory): identical hit counts, CCS within the mixed tolerance."""
    mols, pars = _setup()
    k = len(mols)
    seeds = np.arange(7, 7 + k)
    first = np.full(k, 500, np.int64)
    n = np.full(k, 4000)
    with engine.Batch(mols, pars) as b:
        sums = b.run(seeds, first, n)
        lanes = [b.launch(m)[0] for m in range(k)]
        work, ms = b.counters()
    assert work.steps > 0 and ms > 0
    for m in range(k):
        with engine.Context(mols[m], pars[m], abi.MIXED) as ctx:
            ctx.set_launch(group_lanes=lanes[m])
            s, _, _ = ctx.run_sampled(int(seeds[m]), int(first[m]), int(n[m]))
        assert sums[m].n == s.n and sums[m].n_hit == s.n_hit
        assert abs(sums[m].sum - s.sum) / s.sum < 3e-3


def test_batch_autotune_and_graph_replay():
    mols, pars = _setup()
    k = len(mols)
    with engine.Batch(mols, pars) as b:
        b.autotune()
        seeds, first, n = np.arange(k) + 1, np.zeros(k, np.int64), np.full(k, 2000)
        r1 = b.run(seeds, first, n)
        for m in range(k):
            g, item = b.launch(m)
            assert g in (2, 4, 8, 16, 32) and 0 < item <= 2000   # items sized by cost
        r2 = b.run(seeds, first, n)          # replays the captured graph
        assert [x.sum for x in r1] == [x.sum for x in r2]
        r3 = b.run(seeds, first, n + 17)     # new shape: captured again
        assert all(x.n == 2017 for x in r3)


def test_device_boundary_scan_equals_host(tmp_path):
    """cosims_setup_create_device: the ray march on the GPU gives the host's
    boundary, ellipsoid and path scalars bit for bit."""
    from cosims_b200 import host, synth
    from tests.golden.make_golden import charged128
    for mol, force in ((synth.config1_molecule(), "cutoff"), (charged128(), "multipole12"),
                       (synth.config0_molecule(), "cutoff")):
        mp, ip = synth.write_case(str(tmp_path), mol, force)
        a = host.setup_from_files(mp, ip, seed=1)
        b = host.setup_from_files(mp, ip, seed=1, device=0)
        np.testing.assert_array_equal(a.boundary, b.boundary)
        assert abi.params_to_dict(a.params) == abi.params_to_dict(b.params)


def test_batch_matches_plain_fp64():
    """Each molecule's batched (mixed-form) sums against the plain FP64 form on
    the same sampled trajectories (seed, first index, count): the same hits,
    and the CCS sum within the mixed form's 0.3 % bar at the batched
    configuration's 2e4 trajectories per molecule."""
    mols, pars = _setup()
    k = len(mols)
    seeds = np.arange(31, 31 + k)
    first = np.full(k, 1000, np.int64)
    n = np.full(k, 20000)
    with engine.Batch(mols, pars) as b:
        sums = b.run(seeds, first, n)
    for m in range(k):
        with engine.Context(mols[m], pars[m], abi.PLAIN_F64) as ctx:
            s, _, _ = ctx.run_sampled(int(seeds[m]), int(first[m]), int(n[m]))
        assert sums[m].n == s.n and sums[m].n_hit == s.n_hit
        err = abs(sums[m].sum - s.sum) / s.sum
        print(f"{NAMES[m]}: batched vs plain FP64 CCS sum {100 * err:.3f} %")
        assert err <= 3e-3
