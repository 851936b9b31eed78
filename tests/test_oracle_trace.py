"""The oracle's per-step trace (the checker of cosims_trace_list): the frames
belong to the same trajectories as oracle.run_list's records, one frame per
integration step over all attempts, and the last frame's velocity gives the
recorded scattering angle."""
import numpy as np

from cosims_b200 import abi
from oracle import oracle
from tests.common import hits, load


def test_trace_matches_run_list_and_angle():
    mol, par, d = load("c0_t5")
    p0, v0 = hits(d)
    p0, v0 = p0[:16], v0[:16]
    cap = 4000
    fr, steps, out = oracle.trace(mol, par, p0, v0, cap)
    ref = oracle.run_list(mol, par, p0, v0)
    np.testing.assert_array_equal(out["status"], ref["status"])
    np.testing.assert_array_equal(out["chi"], ref["chi"])
    np.testing.assert_array_equal(out["steps"], ref["steps"])
    retries = ((out["status"] >> abi.TRAJ_ETRIES_SHIFT) & 0xff) + \
              ((out["status"] >> abi.TRAJ_OTRIES_SHIFT) & 0xff)
    plain = retries == 0
    assert plain.any()
    # without retries every step of the one attempt is a frame
    np.testing.assert_array_equal(steps[plain], out["steps"][plain])
    assert (steps >= out["steps"]).all() and (steps <= cap).all()
    ok = plain & ((out["status"] & abi.TRAJ_SUCCESS) > 0)
    for i in np.nonzero(ok)[0]:
        v = fr[i, steps[i] - 1, 3:]
        c = np.dot(v0[i], v) / (np.linalg.norm(v0[i]) * np.linalg.norm(v))
        assert abs(np.arccos(np.clip(c, -1, 1)) - out["chi"][i]) < 1e-9


def test_trace_respects_the_frame_cap():
    mol, par, d = load("c0_t5")
    p0, v0 = hits(d)
    fr, steps, out = oracle.trace(mol, par, p0[:4], v0[:4], 5)
    assert fr.shape == (4, 5, 6)
    assert (steps > 5).all()
    full, _, _ = oracle.trace(mol, par, p0[:4], v0[:4], 50)
    np.testing.assert_array_equal(fr, full[:, :5])
