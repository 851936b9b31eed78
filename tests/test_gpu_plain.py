"""Plain FP64 form on the GPU against the reference (golden fixtures) and the
oracle.  The plain kernel keeps the reference's IEEE operation order, so
trajectories match bit for bit; only the final acos of chi may differ in the
last ulp (CUDA's acos vs glibc's).  Tolerance: |d chi| <= 1e-12 rad, identical
success flags, step counts and energy deviations within 1e-12 relative."""
import numpy as np
import pytest

from cosims_b200 import abi, engine
from oracle import oracle
from tests.common import CASES, hits, load

pytestmark = pytest.mark.gpu

CHI_TOL = 1e-12


def _check(out, chi, succ, steps, de):
    assert np.max(np.abs(out["chi"] - chi)) <= CHI_TOL
    np.testing.assert_array_equal((out["status"] & abi.TRAJ_SUCCESS) > 0, succ)
    np.testing.assert_array_equal(out["steps"], steps)
    np.testing.assert_allclose(out["de_pct"], de, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("name", CASES)
def test_plain_matches_reference(name):
    mol, par, d = load(name)
    p0, v0 = hits(d)
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        out = ctx.run_list(p0, v0)
    _check(out, d["ref_chi"], d["ref_succ"] == 1, d["ref_steps"], d["ref_de"])


@pytest.mark.parametrize("name", CASES)
def test_plain_handoff_is_bit_exact(name):
    """With a step budget of 16 nearly every trajectory is parked and finished
    by a whole CTA that adds the terms in the serial order: the results must be
    the reference's bit for bit, as without the hand-off."""
    mol, par, d = load(name)
    p0, v0 = hits(d)
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        ctx.set_handoff(16, 0)
        out = ctx.run_list(p0, v0)
        parked = ctx.get_handoff()[2]
        ctx.set_handoff(-1, 0)
        off = ctx.run_list(p0, v0)
    assert parked > len(p0) // 2
    _check(out, d["ref_chi"], d["ref_succ"] == 1, d["ref_steps"], d["ref_de"])
    np.testing.assert_array_equal(out, off)


@pytest.mark.parametrize("name", ["c0_t5", "q128_t1", "q128_t4", "c1_t3"])
def test_plain_matches_oracle_on_device_sampled_inputs(name):
    """Sampled start states from the device; same states through the oracle."""
    mol, par, _ = load(name)
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        ins, pos0, vel0, hit = ctx.sample_inputs(seed=11, first=0, n=400)
        sel = hit == 1
        out = ctx.run_list(pos0[sel], vel0[sel])
    ref = oracle.run_list(mol, par, pos0[sel], vel0[sel])
    _check(out, ref["chi"], (ref["status"] & abi.TRAJ_SUCCESS) > 0, ref["steps"], ref["de_pct"])
    np.testing.assert_array_equal(out["status"], ref["status"])


def test_plain_empty_and_single():
    mol, par, d = load("c0_t5")
    p0, v0 = hits(d)
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        assert ctx.run_list(p0[:0], v0[:0]).shape == (0,)
        one = ctx.run_list(p0[:1], v0[:1])
    assert abs(one["chi"][0] - d["ref_chi"][0]) <= CHI_TOL


def test_plain_step_cap_reports_failure():
    """A trajectory stopped by max_steps is a failure with chi = pi/2."""
    mol, par, d = load("c0_t5")
    p0, v0 = hits(d)
    par.max_steps = 20
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        out = ctx.run_list(p0[:64], v0[:64])
    ref = oracle.run_list(mol, par, p0[:64], v0[:64])
    np.testing.assert_array_equal(out["status"], ref["status"])
    capped = (out["status"] & abi.TRAJ_STEPCAP) > 0
    assert capped.any()
    assert np.all(out["chi"][capped] == np.pi / 2)


@pytest.mark.parametrize("name", ["c0_t5", "q128_t1", "c1_t3"])
def test_trace_equals_oracle_trace(name):
    """cosims_trace_list: the position and velocity after every step, bit for
    bit the oracle's (all attempts), and the same results as run_list."""
    mol, par, d = load(name)
    p0, v0 = hits(d)
    p0, v0 = p0[:24], v0[:24]
    cap = 200                                   # some trajectories run past it
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        fr, steps, out = ctx.trace_list(p0, v0, cap)
        plain = ctx.run_list(p0, v0)
        _, steps0, out0 = ctx.trace_list(p0, v0, 0)
    rfr, rsteps, rout = oracle.trace(mol, par, p0, v0, cap)
    np.testing.assert_array_equal(steps, rsteps)
    np.testing.assert_array_equal(steps0, rsteps)
    assert (steps > cap).any() and (steps <= cap).any()
    np.testing.assert_array_equal(fr, rfr)
    for o in (out, out0):
        np.testing.assert_array_equal(o["status"], plain["status"])
        np.testing.assert_array_equal(o["chi"], plain["chi"])
        np.testing.assert_array_equal(o["steps"], plain["steps"])


def test_trace_needs_the_plain_form():
    mol, par, d = load("c0_t5")
    p0, v0 = hits(d)
    with engine.Context(mol, par, abi.MIXED) as ctx:
        with pytest.raises(engine.CosimsError):
            ctx.trace_list(p0[:2], v0[:2], 10)
