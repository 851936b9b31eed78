"""cosims_run_list_noalloc: the trajectory run for callers that cannot let the
library allocate device memory (a host program with its own GPU memory pool,
or one that forbids cudaMalloc on its hot path).  The caller allocates the
start states and the result buffer; the library keeps its scratch in a
static device array.  Its results must equal the context path's
(cosims_run_list) within the tolerance of the plain-form tests, on two calls
in a row (the second call reuses the array the first one left behind).

Collected last on purpose (file name), so that a run stopping at the first
failure has run every other test already."""
import ctypes as C

import numpy as np
import pytest

from cosims_b200 import abi, engine
from tests.common import hits, load

pytestmark = pytest.mark.gpu

CHI_TOL = 1e-12          # as tests/test_gpu_plain.py
MAX_TRAJ = 2_096_128     # the documented per-call limit


def _noalloc():
    f = engine.lib().cosims_run_list_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.Molecule), C.POINTER(abi.Params), C.c_int32, C.c_int32,
                  C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    return f


@pytest.mark.parametrize("name,precision,lanes", [("q128_t1", abi.PLAIN_F64, 1),
                                                  ("c1_t3", abi.MIXED, 8),
                                                  ("c0_t5", abi.MIXED, 4)])
def test_noalloc_matches_context_path_twice(name, precision, lanes):
    import torch
    mol, par, d = load(name)
    p0, v0 = hits(d)
    n = p0.shape[0]
    with engine.Context(mol, par, precision) as ctx:
        if precision == abi.MIXED:
            ctx.set_launch(group_lanes=lanes)
        ref = ctx.run_list(p0, v0)
    dp0 = torch.from_numpy(np.ascontiguousarray(p0)).cuda()
    dv0 = torch.from_numpy(np.ascontiguousarray(v0)).cuda()
    dout = torch.empty(n * abi.TRAJ_OUT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    view = mol.view()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    f = _noalloc()
    for call in range(2):
        dout.fill_(0xA5)                      # stale bytes must all be overwritten
        engine.check(f(C.byref(view), C.byref(par), precision, lanes, dp0.data_ptr(),
                       dv0.data_ptr(), n, dout.data_ptr(), stream))
        torch.cuda.synchronize()
        out = np.frombuffer(dout.cpu().numpy().tobytes(), dtype=abi.TRAJ_OUT_DTYPE)
        assert np.max(np.abs(out["chi"] - ref["chi"])) <= CHI_TOL, f"call {call}"
        np.testing.assert_array_equal(out["status"], ref["status"])
        np.testing.assert_array_equal(out["steps"], ref["steps"])
        np.testing.assert_allclose(out["de_pct"], ref["de_pct"], rtol=1e-12, atol=1e-14)


def test_noalloc_rejects_sizes_beyond_its_limit():
    mol, par, _ = load("c0_t5")
    view = mol.view()
    rc = _noalloc()(C.byref(view), C.byref(par), abi.PLAIN_F64, 1, None, None, MAX_TRAJ + 1,
                    None, None)
    assert rc == abi.ERR_UNSUPPORTED
    assert b"no-alloc limit" in engine.lib().cosims_last_error()


def test_noalloc_rejects_a_molecule_image_beyond_its_limit():
    """16000 atoms in 16000 one-atom clusters need about 7 MB of images, more
    than the 4 MiB the array holds for them."""
    mol, par, _ = load("c0_t5")
    n = 16000
    rng = np.random.default_rng(3)
    xyz = rng.normal(0.0, 30.0, size=(n, 3))
    big = abi.MoleculeArrays(
        xyz=xyz, charge=np.zeros(n), sig6=np.full(n, mol.sig6[1]),
        eps24m=np.full(n, mol.eps24m[1]), eps4=np.full(n, mol.eps4[1]),
        cluster_offset=np.arange(n + 1, dtype=np.int32),
        cluster_atoms=np.arange(n, dtype=np.int32), cluster_pos=xyz,
        cluster_radius=np.zeros(n), cluster_charge=np.zeros(n),
        cluster_dipole=np.zeros((n, 3)), cluster_quad=np.zeros((n, 9)),
        cluster_replaced=np.zeros(n, np.int32))
    view = big.view()
    rc = _noalloc()(C.byref(view), C.byref(par), abi.PLAIN_F64, 1, None, None, 0, None, None)
    assert rc == abi.ERR_UNSUPPORTED
    assert b"no-alloc limit" in engine.lib().cosims_last_error()


def test_noalloc_runs_without_handoff():
    """The path has no long-trajectory hand-off.  On a mixed-form list that
    holds trajectories past the context's 2048-step budget, its results are bit
    for bit those of a context with the hand-off off."""
    import torch
    mol, par, _ = load("c1_t3")
    lanes = 8
    with engine.Context(mol, par, abi.MIXED) as ctx:
        ctx.set_launch(group_lanes=lanes)
        ctx.set_handoff(-1, 0)
        _, p0, v0, hit = ctx.sample_inputs(seed=2, first=0, n=40000)
        p0, v0 = p0[hit == 1], v0[hit == 1]
        scan = ctx.run_list(p0, v0)
        long_ = np.flatnonzero(scan["steps"] > 2048)
        assert long_.size > 0, "no trajectory past 2048 steps in the sample"
        sel = np.concatenate([np.arange(300), long_])
        p0, v0 = np.ascontiguousarray(p0[sel]), np.ascontiguousarray(v0[sel])
        ref = ctx.run_list(p0, v0)
    n = p0.shape[0]
    dp0 = torch.from_numpy(p0).cuda()
    dv0 = torch.from_numpy(v0).cuda()
    dout = torch.empty(n * abi.TRAJ_OUT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    view = mol.view()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    engine.check(_noalloc()(C.byref(view), C.byref(par), abi.MIXED, lanes, dp0.data_ptr(),
                            dv0.data_ptr(), n, dout.data_ptr(), stream))
    torch.cuda.synchronize()
    out = np.frombuffer(dout.cpu().numpy().tobytes(), dtype=abi.TRAJ_OUT_DTYPE)
    np.testing.assert_array_equal(out, ref)
    assert (out["steps"] > 2048).any()
