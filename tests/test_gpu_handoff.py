"""Long-trajectory hand-off of the mixed form.

A trajectory still running after the step budget is parked and finished by a
wide group (one trajectory per wide_lanes threads).  Bars: results are a
function of the trajectory and the settings alone (bitwise the same on a
rerun, whatever runs beside it); hits are identical to the no-hand-off run;
CCS within the mixed tolerance (0.3 %) of the plain FP64 form; every parked
trajectory gets its record."""
import numpy as np
import pytest

from cosims_b200 import abi, engine
from tests.common import load

pytestmark = pytest.mark.gpu

CCS_TOL = 3e-3


def _run(name, n, budget, wide, lanes=8, first=0):
    mol, par, _ = load(name)
    with engine.Context(mol, par, abi.MIXED) as ctx:
        ctx.set_launch(group_lanes=lanes)
        ctx.set_handoff(budget, wide)
        s, ins, outs = ctx.run_sampled(99, first, n, want_records=True)
        return s, outs, ctx.get_handoff()


@pytest.mark.parametrize("name,wide", [("c1_t3", 128), ("q128_t1", 64), ("c0_t5", 32),
                                       ("c2_t1", 256)])
def test_handoff_deterministic_and_complete(name, wide):
    n = 4000 if name != "c2_t1" else 1000
    s1, o1, h1 = _run(name, n, 64, wide)
    s2, o2, h2 = _run(name, n, 64, wide)
    assert h1[2] > 0 and h1[3] > 0            # trajectories were parked and finished wide
    assert np.array_equal(o1, o2)             # bitwise the same on a rerun
    assert (s1.sum, s1.n_eff, s1.steps) == (s2.sum, s2.n_eff, s2.steps)
    s0, o0, h0 = _run(name, n, -1, 0)
    assert h0[2] == 0
    # a parked trajectory left without a record would read as a miss here
    hit = (o0["status"] & abi.TRAJ_HIT) > 0
    assert np.array_equal(hit, (o1["status"] & abi.TRAJ_HIT) > 0)


@pytest.mark.parametrize("name,n", [("c1_t3", 20000), ("q128_t4", 20000)])
def test_handoff_ccs_within_tolerance_of_plain(name, n):
    mol, par, _ = load(name)
    with engine.Context(mol, par, abi.PLAIN_F64) as cp:
        sp, _, _ = cp.run_sampled(5, 0, n)
    for budget, wide in [(32, 128), (1024, 128), (256, 32)]:
        with engine.Context(mol, par, abi.MIXED) as cm:
            cm.set_handoff(budget, wide)
            sm, _, _ = cm.run_sampled(5, 0, n)
        assert sm.n == sp.n and sm.n_hit == sp.n_hit
        assert abs(sm.sum - sp.sum) / sp.sum < CCS_TOL


def test_handoff_settings_validated():
    mol, par, _ = load("q128_t1")
    with engine.Context(mol, par, abi.MIXED) as cm:
        with pytest.raises(engine.CosimsError):
            cm.set_handoff(0, 48)                # not a multiple of 32
        cm.set_handoff(0, 0)
        assert cm.get_handoff()[0] == 2048       # default budget
    with engine.Context(mol, par, abi.PLAIN_F64) as cp:
        with pytest.raises(engine.CosimsError):
            cp.set_handoff(100, 64)              # the plain form's wide group is its CTA
        cp.set_handoff(0, 0)
        assert cp.get_handoff()[0] == 256        # the plain form's default budget
