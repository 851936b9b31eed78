"""The error path on the GPU, made without any fault.

Every device wait of the trajectory kernels is bounded.  A wait that gives up
sets an error flag and the kernel returns; the call then returns
COSIMS_ERR_TIMEOUT and the context stays usable.  cosims_ctx_set_wait_test
makes a wait give up on purpose: the staging wait at once (the CTA still waits
for its copies in flight before it leaves), or the hand-off wait on a record
flag that nothing sets.  The reference's own failure branch -- a trajectory
whose energy check fails on every retry (diffEqSolver.cpp:139-210) -- is
reproduced with a time step far too large to conserve energy."""
import numpy as np
import pytest

from cosims_b200 import abi, engine
from oracle import oracle
from tests.common import hits, load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [abi.PLAIN_F64, abi.MIXED])
def test_staging_wait_gives_up_and_context_recovers(precision):
    # the 128-atom molecule: both forms stage its image in shared memory
    mol, par, d = load("c0_t5")
    p0, v0 = hits(d)
    with engine.Context(mol, par, precision) as ctx:
        good = ctx.run_list(p0, v0)
        ctx.set_wait_test(abi.WAIT_TEST_STAGING)
        with pytest.raises(engine.CosimsError) as ei:
            ctx.run_list(p0, v0)
        assert ei.value.status == abi.ERR_TIMEOUT
        assert "staging" in str(ei.value)
        ctx.set_wait_test(0)
        again = ctx.run_list(p0, v0)
    np.testing.assert_array_equal(good, again)


@pytest.mark.parametrize("precision", [abi.PLAIN_F64, abi.MIXED])
def test_handoff_wait_gives_up_and_context_recovers(precision):
    """With a 16-step budget most trajectories are parked; the first parked
    record is never published, so the wide group that takes it gives up after
    4096 polls.  The others still finish."""
    mol, par, d = load("c0_t5")
    p0, v0 = hits(d)
    with engine.Context(mol, par, precision) as ctx:
        ctx.set_handoff(16, 0)
        good = ctx.run_list(p0, v0)
        ctx.set_wait_test(abi.WAIT_TEST_HANDOFF, 4096)
        with pytest.raises(engine.CosimsError) as ei:
            ctx.run_list(p0, v0)
        assert ei.value.status == abi.ERR_TIMEOUT
        assert "hand-off" in str(ei.value)
        ctx.set_wait_test(0)
        again = ctx.run_list(p0, v0)
    np.testing.assert_array_equal(good, again)


def test_wait_test_rejects_unknown_flags():
    mol, par, _ = load("c0_t5")
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        with pytest.raises(engine.CosimsError) as ei:
            ctx.set_wait_test(0x80)
        assert ei.value.status == abi.ERR_INVALID


def test_energy_check_fails_every_retry_like_the_reference():
    """dt = 0.5 ps (50x the default) cannot keep the energy within 0.5 % on
    close collisions: those trajectories fail after their energy retries with
    chi = pi/2, exactly as the oracle's verletVel restatement says, retry
    counts included."""
    mol, par, d = load("q128_t3")
    p0, v0 = hits(d)
    p0, v0 = p0[:64], v0[:64]
    par.dt = 0.5
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        out = ctx.run_list(p0, v0)
    ref = oracle.run_list(mol, par, p0, v0)
    np.testing.assert_array_equal(out["status"], ref["status"])
    np.testing.assert_array_equal(out["steps"], ref["steps"])
    assert np.max(np.abs(out["chi"] - ref["chi"])) <= 1e-12
    failed = (out["status"] & abi.TRAJ_SUCCESS) == 0
    assert failed.sum() >= 4
    assert np.all(out["chi"][failed] == np.pi / 2)
    etries = (out["status"] >> abi.TRAJ_ETRIES_SHIFT) & 0xff
    assert etries[failed].max() >= 1
