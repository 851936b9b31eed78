"""A near collision in the mixed form: a pair term that overflows FP32 leaves
a non-finite state where the reference's FP64 state holds a huge, finite
energy error.  The energy check must fail it and retry with a smaller time
step (diffEqSolver.cpp:188-194), not record a success with chi = NaN.

Trajectory 1 332 039 of the 3000-atom protein workload (seed 20251203, 32
lanes per trajectory) is such a case: before the check treated a non-finite
energy as a failure, it ended as a success with chi = NaN and turned the
integral's CCS into NaN."""
import tempfile

import numpy as np
import pytest

from cosims_b200 import abi, engine, host, synth

pytestmark = pytest.mark.gpu

SEED = 20251203


@pytest.fixture(scope="module")
def protein():
    tmp = tempfile.mkdtemp(prefix="cosims_protein_")
    mp, ip = synth.write_case(tmp, synth.config2_molecule(), "multipole12",
                              traj_thousands=1000, iterations=1)
    st = host.setup_from_files(mp, ip, seed=SEED, device=0)
    return st.mol, st.params


def test_near_collision_retries_instead_of_nan(protein):
    mol, par = protein
    with engine.Context(mol, par, abi.MIXED) as ctx:
        ctx.set_launch(group_lanes=32)
        s, _, out = ctx.run_sampled(SEED, 1_332_039, 1, want_records=True)
        assert np.isfinite(out["chi"]).all() and np.isfinite(out["de_pct"]).all()
        # its neighbourhood of the stream, and the integral's sums
        s, _, out = ctx.run_sampled(SEED, 1_320_000, 20_000, want_records=True)
    assert np.isfinite(out["chi"]).all() and np.isfinite(out["de_pct"]).all()
    assert np.isfinite(s.sum) and np.isfinite(s.sum2) and s.n_eff > 0
