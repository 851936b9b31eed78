"""Python binding of the CCS engine's C ABI (include/cosims_cuda.h).

`Context` mirrors the reference's per-molecule trajectory driver (monteTraj,
monteTraj.cpp:26-502): it owns one molecule on the device and runs batches of
trajectories through the CUDA kernels.  There is no CPU path: if the CUDA
library or a B200 is missing, every call raises `CosimsError`.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libcosims_cuda.so")

_LIB = None
_LOCK = threading.Lock()


class CosimsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"cosims status {status}: {message}")
        self.status = status


def lib():
    """Load libcosims_cuda.so (built by cosims_b200.build.build())."""
    global _LIB
    with _LOCK:
        if _LIB is None:
            if not os.path.exists(LIB_PATH):
                raise CosimsError(abi.ERR_UNSUPPORTED,
                                  f"CUDA library missing: {LIB_PATH} (run the build)")
            L = C.CDLL(LIB_PATH)
            P, V = C.POINTER, C.c_void_p
            st = C.c_int
            sig = {
                "cosims_abi_version": (C.c_int32, []),
                "cosims_last_error": (C.c_char_p, []),
                "cosims_device_count": (C.c_int32, []),
                "cosims_ctx_create": (st, [P(abi.Molecule), P(abi.Params), C.c_int32, C.c_int32,
                                           P(V)]),
                "cosims_ctx_destroy": (None, [V]),
                "cosims_ctx_set_launch": (st, [V, C.c_int32, C.c_int32]),
                "cosims_ctx_get_launch": (st, [V, P(C.c_int32), P(C.c_int32)]),
                "cosims_run_list": (st, [V, V, V, C.c_int64, V, V]),
                "cosims_run_list_device": (st, [V, V, V, C.c_int64, V, V]),
                "cosims_trace_list": (st, [V, V, V, C.c_int64, C.c_int32, V, V, V, V]),
                "cosims_run_sampled": (st, [V, C.c_uint64, C.c_int64, C.c_int64, C.c_int64,
                                            P(abi.CcsSums), V, V, V]),
                "cosims_run_sampled_device": (st, [V, C.c_uint64, C.c_int64, C.c_int64,
                                                   C.c_int64, V, V]),
                "cosims_sample_inputs": (st, [V, C.c_uint64, C.c_int64, C.c_int64, V, V, V, V,
                                              V]),
                "cosims_run_integrals": (st, [V, C.c_uint64, C.c_int64, C.c_int64, C.c_int32,
                                              C.c_int64, V, V, V]),
                "cosims_run_integrals_device": (st, [V, C.c_uint64, C.c_int64, C.c_int64,
                                                     C.c_int32, C.c_int64, V, V, V]),
                "cosims_batch_create": (st, [V, V, C.c_int32, C.c_int32, C.c_int32, P(V)]),
                "cosims_batch_destroy": (None, [V]),
                "cosims_batch_autotune": (st, [V, V]),
                "cosims_batch_run": (st, [V, V, V, V, V, V]),
                "cosims_batch_run_async": (st, [V, V, V, V, V, V]),
                "cosims_batch_get_launch": (st, [V, C.c_int32, P(C.c_int32), P(C.c_int32)]),
                "cosims_batch_set_update_every": (st, [V, C.c_int64]),
                "cosims_batch_counters": (st, [V, P(abi.CcsSums), P(C.c_float)]),
                "cosims_ctx_kernel_ms": (st, [V, P(C.c_float)]),
                "cosims_ctx_kernel_timeline": (st, [V, P(C.c_double), P(C.c_double)]),
                "cosims_ctx_set_handoff": (st, [V, C.c_int64, C.c_int32]),
                "cosims_ctx_reserve": (st, [V, C.c_int64, C.c_int32]),
                "cosims_ctx_set_wait_test": (st, [V, C.c_uint32, C.c_uint32]),
                "cosims_ctx_get_handoff": (st, [V, P(C.c_int64), P(C.c_int32), P(C.c_int64),
                                                P(C.c_int64), P(C.c_double)]),
                "cosims_serve_create": (st, [C.c_int32, C.c_int64, C.c_int32, C.c_int64, P(V)]),
                "cosims_serve_destroy": (None, [V]),
                "cosims_serve_submit": (st, [V, P(abi.Molecule), P(abi.Params), C.c_uint64,
                                             C.c_double, C.c_int64, C.c_int64, P(C.c_int64)]),
                "cosims_serve_step": (st, [V, V, P(C.c_int32)]),
                "cosims_serve_poll": (st, [V, C.c_int64, P(abi.JobStatus)]),
                "cosims_serve_release": (st, [V, C.c_int64]),
                "cosims_serve_info": (st, [V, P(C.c_int32), P(C.c_int64)]),
                "cosims_serve_set_max_chunk": (st, [V, C.c_int64]),
                "cosims_probe_peaks": (st, [C.c_int32, P(C.c_double), P(C.c_double)]),
            }
            for name, (res, args) in sig.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            if L.cosims_abi_version() != abi.ABI_VERSION:
                raise CosimsError(abi.ERR_UNSUPPORTED, "ABI version mismatch")
            _LIB = L
    return _LIB


def check(status: int) -> None:
    if status != abi.OK:
        msg = lib().cosims_last_error()
        raise CosimsError(status, msg.decode() if msg else "")


def device_count() -> int:
    return int(lib().cosims_device_count())


def _stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(int(stream.cuda_stream))     # torch.cuda.Stream


class Context:
    """One molecule resident on the device (plain FP64 or mixed precision)."""

    def __init__(self, mol: abi.MoleculeArrays, par: abi.Params,
                 precision: int = abi.PLAIN_F64, device: int = 0):
        self.mol = mol
        self.par = par
        self.precision = precision
        self.device = device
        self._view = mol.view()
        h = C.c_void_p()
        check(lib().cosims_ctx_create(C.byref(self._view), C.byref(par), precision, device,
                                      C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().cosims_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def set_launch(self, group_lanes: int = 0, block_threads: int = 0) -> None:
        check(lib().cosims_ctx_set_launch(self._h, group_lanes, block_threads))

    def get_launch(self) -> tuple:
        g, b = C.c_int32(), C.c_int32()
        check(lib().cosims_ctx_get_launch(self._h, C.byref(g), C.byref(b)))
        return g.value, b.value

    def run_list(self, pos0: np.ndarray, vel0: np.ndarray, stream=None,
                 out: np.ndarray | None = None) -> np.ndarray:
        """verletVel on each start state; returns TRAJ_OUT_DTYPE records
        (written into `out` when given, e.g. a pinned host array)."""
        pos0 = np.ascontiguousarray(pos0, dtype=np.float64).reshape(-1, 3)
        vel0 = np.ascontiguousarray(vel0, dtype=np.float64).reshape(-1, 3)
        if out is None:
            out = np.zeros(pos0.shape[0], dtype=abi.TRAJ_OUT_DTYPE)
        elif out.dtype != abi.TRAJ_OUT_DTYPE or out.shape[0] < pos0.shape[0] or \
                not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous TRAJ_OUT_DTYPE array of n records")
        check(lib().cosims_run_list(self._h, abi.vptr(pos0), abi.vptr(vel0), pos0.shape[0],
                                    abi.vptr(out), _stream_ptr(stream)))
        return out

    def trace_list(self, pos0: np.ndarray, vel0: np.ndarray, max_frames: int, stream=None):
        """Plain form: verletVel on each start state, recording position and
        velocity after every step.  Returns (frames [n, max_frames, 6],
        steps integrated [n], TRAJ_OUT_DTYPE records); frames[i, :min(steps[i],
        max_frames)] are trajectory i's."""
        pos0 = np.ascontiguousarray(pos0, dtype=np.float64).reshape(-1, 3)
        vel0 = np.ascontiguousarray(vel0, dtype=np.float64).reshape(-1, 3)
        n = pos0.shape[0]
        frames = np.zeros((n, max_frames, 6))
        steps = np.zeros(n, dtype=np.int32)
        out = np.zeros(n, dtype=abi.TRAJ_OUT_DTYPE)
        check(lib().cosims_trace_list(self._h, abi.vptr(pos0), abi.vptr(vel0), n, int(max_frames),
                                      abi.vptr(frames) if max_frames else None, abi.vptr(steps),
                                      abi.vptr(out), _stream_ptr(stream)))
        return frames, steps, out

    def run_list_device(self, d_pos0: int, d_vel0: int, n: int, d_out: int, stream=None) -> None:
        check(lib().cosims_run_list_device(self._h, C.c_void_p(d_pos0), C.c_void_p(d_vel0), n,
                                           C.c_void_p(d_out), _stream_ptr(stream)))

    def run_sampled(self, seed: int, first: int, n: int, update_every: int = 0,
                    want_records: bool = False, stream=None):
        """One CCS integral of n sampled trajectories.  Returns (sums, inputs, outs)."""
        s = abi.CcsSums()
        ins = np.zeros(n, abi.TRAJ_IN_DTYPE) if want_records else None
        outs = np.zeros(n, abi.TRAJ_OUT_DTYPE) if want_records else None
        check(lib().cosims_run_sampled(
            self._h, seed, first, n, update_every, C.byref(s),
            abi.vptr(ins) if ins is not None else None,
            abi.vptr(outs) if outs is not None else None, _stream_ptr(stream)))
        return s, ins, outs

    def run_sampled_device(self, seed: int, first: int, n: int, update_every: int,
                           d_sums: int, stream=None) -> None:
        check(lib().cosims_run_sampled_device(self._h, seed, first, n, update_every,
                                              C.c_void_p(d_sums), _stream_ptr(stream)))

    def run_integrals(self, seed: int, first: int, n_per: int, n_integrals: int,
                      update_every: int = 0, stream=None) -> tuple:
        """n_integrals CCS integrals of n_per trajectories each (integral k is
        trajectories first + k * n_per ...), in as few launches as possible.
        Returns (list of per-integral sums, the call's work counters)."""
        recs = (abi.CcsSums * max(n_integrals, 1))()
        work = abi.CcsSums()
        check(lib().cosims_run_integrals(self._h, seed, first, n_per, n_integrals, update_every,
                                         C.cast(recs, C.c_void_p), C.byref(work),
                                         _stream_ptr(stream)))
        return [recs[k] for k in range(n_integrals)], work

    def run_integrals_device(self, seed: int, first: int, n_per: int, n_integrals: int,
                             update_every: int, d_sums: int, d_work: int = 0,
                             stream=None) -> None:
        check(lib().cosims_run_integrals_device(self._h, seed, first, n_per, n_integrals,
                                                update_every, C.c_void_p(d_sums),
                                                C.c_void_p(d_work) if d_work else None,
                                                _stream_ptr(stream)))

    def reserve(self, n_traj: int, n_integrals: int = 1) -> None:
        """Allocate the buffers of calls of up to n_traj trajectories (and up to
        n_integrals integrals per run_integrals call) now, not in the calls."""
        check(lib().cosims_ctx_reserve(self._h, int(n_traj), int(n_integrals)))

    def set_wait_test(self, flags: int = 0, spin_limit: int = 0) -> None:
        """Make the bounded device waits give up on purpose (tests of the
        error path; abi.WAIT_TEST_* flags, 0 restores normal runs)."""
        check(lib().cosims_ctx_set_wait_test(self._h, int(flags), int(spin_limit)))

    def kernel_ms(self) -> float:
        """Device time of the last trajectory-kernel launch (CUDA events)."""
        ms = C.c_float()
        check(lib().cosims_ctx_kernel_ms(self._h, C.byref(ms)))
        return ms.value

    def set_handoff(self, step_budget: int = 0, wide_lanes: int = 0) -> None:
        """Park trajectories after step_budget steps (0 default, < 0 off) and
        finish them in wide groups: wide_lanes threads in the mixed form, the
        whole 128-thread CTA in the plain form (bitwise the same results)."""
        check(lib().cosims_ctx_set_handoff(self._h, int(step_budget), int(wide_lanes)))

    def get_handoff(self) -> tuple:
        """(step_budget, wide_lanes, parked, wide_steps, wide_ms) of the last run."""
        b, w, n = C.c_int64(), C.c_int32(), C.c_int64()
        ws, wm = C.c_int64(), C.c_double()
        check(lib().cosims_ctx_get_handoff(self._h, C.byref(b), C.byref(w), C.byref(n),
                                           C.byref(ws), C.byref(wm)))
        return b.value, w.value, n.value, ws.value, wm.value

    def kernel_timeline(self) -> tuple:
        """(drain_ms, end_ms) of the last trajectory kernel: when a group first
        found the work queue empty, and when the last group exited."""
        d, e = C.c_double(), C.c_double()
        check(lib().cosims_ctx_kernel_timeline(self._h, C.byref(d), C.byref(e)))
        return d.value, e.value

    def sample_inputs(self, seed: int, first: int, n: int, stream=None):
        ins = np.zeros(n, abi.TRAJ_IN_DTYPE)
        pos0, vel0 = np.zeros((n, 3)), np.zeros((n, 3))
        hit = np.zeros(n, np.int32)
        check(lib().cosims_sample_inputs(self._h, seed, first, n, abi.vptr(ins), abi.vptr(pos0),
                                         abi.vptr(vel0), abi.vptr(hit), _stream_ptr(stream)))
        return ins, pos0, vel0, hit


class Batch:
    """Many molecules in one persistent launch (mixed precision)."""

    def __init__(self, mols: list, pars: list, device: int = 0):
        self.mols = mols
        self.pars = pars
        self.device = device
        self._views = (abi.Molecule * len(mols))(*[m.view() for m in mols])
        self._pars = (abi.Params * len(pars))(*pars)
        h = C.c_void_p()
        check(lib().cosims_batch_create(C.cast(self._views, C.c_void_p),
                                        C.cast(self._pars, C.c_void_p), len(mols), abi.MIXED,
                                        device, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().cosims_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def autotune(self, stream=None) -> None:
        check(lib().cosims_batch_autotune(self._h, _stream_ptr(stream)))

    def launch(self, mol: int) -> tuple:
        g, it = C.c_int32(), C.c_int32()
        check(lib().cosims_batch_get_launch(self._h, mol, C.byref(g), C.byref(it)))
        return g.value, it.value

    def set_update_every(self, k: int) -> None:
        check(lib().cosims_batch_set_update_every(self._h, int(k)))

    def run(self, seeds, firsts, n_traj, stream=None) -> list:
        k = len(self.mols)
        sd = np.ascontiguousarray(seeds, dtype=np.uint64)
        fi = np.ascontiguousarray(firsts, dtype=np.int64)
        nt = np.ascontiguousarray(n_traj, dtype=np.int64)
        out = (abi.CcsSums * k)()
        check(lib().cosims_batch_run(self._h, abi.vptr(sd), abi.vptr(fi), abi.vptr(nt),
                                     C.cast(out, C.c_void_p), _stream_ptr(stream)))
        return list(out)

    def run_async(self, seeds, firsts, n_traj, d_sums: int = 0, stream=None) -> None:
        sd = np.ascontiguousarray(seeds, dtype=np.uint64)
        fi = np.ascontiguousarray(firsts, dtype=np.int64)
        nt = np.ascontiguousarray(n_traj, dtype=np.int64)
        check(lib().cosims_batch_run_async(self._h, abi.vptr(sd), abi.vptr(fi), abi.vptr(nt),
                                           C.c_void_p(d_sums), _stream_ptr(stream)))

    def counters(self) -> tuple:
        w, ms = abi.CcsSums(), C.c_float()
        check(lib().cosims_batch_counters(self._h, C.byref(w), C.byref(ms)))
        return w, ms.value


class Server:
    """Continuous-batching CCS service: jobs admitted by HBM footprint, each
    molecule and its running sums resident on the device until released."""

    def __init__(self, device: int = 0, hbm_budget: int = 8 << 30, max_jobs: int = 64,
                 round_traj: int = 16384):
        h = C.c_void_p()
        check(lib().cosims_serve_create(device, int(hbm_budget), int(max_jobs), int(round_traj),
                                        C.byref(h)))
        self._h = h
        self.round_traj = round_traj
        self._keep = {}

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().cosims_serve_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, mol: abi.MoleculeArrays, par: abi.Params, seed: int, target_rel_se: float,
               min_traj: int = 0, max_traj: int = 1 << 40):
        """Job id, or None when the server has no room now (admission)."""
        view = mol.view()
        jid = C.c_int64()
        st = lib().cosims_serve_submit(self._h, C.byref(view), C.byref(par), int(seed),
                                       float(target_rel_se), int(min_traj), int(max_traj),
                                       C.byref(jid))
        if st == abi.ERR_BUSY:
            return None
        check(st)
        return jid.value

    def step(self, stream=None) -> int:
        n = C.c_int32()
        check(lib().cosims_serve_step(self._h, _stream_ptr(stream), C.byref(n)))
        return n.value

    def poll(self, job_id: int) -> abi.JobStatus:
        s = abi.JobStatus()
        check(lib().cosims_serve_poll(self._h, job_id, C.byref(s)))
        return s

    def release(self, job_id: int) -> None:
        check(lib().cosims_serve_release(self._h, job_id))

    def set_max_chunk(self, max_chunk_traj: int) -> None:
        """Largest chunk of one job in one round (0: the default, 64 round_traj)."""
        check(lib().cosims_serve_set_max_chunk(self._h, int(max_chunk_traj)))

    def info(self) -> tuple:
        a, b = C.c_int32(), C.c_int64()
        check(lib().cosims_serve_info(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value


def probe_peaks(device: int = 0) -> tuple:
    """Measured FP32 and FP64 FMA throughput of the device, TFLOP/s."""
    f32, f64 = C.c_double(), C.c_double()
    check(lib().cosims_probe_peaks(device, C.byref(f32), C.byref(f64)))
    return f32.value, f64.value


def omega(s: abi.CcsSums) -> tuple:
    """Omega and its standard error for one integral (monteTraj.cpp:381-387)."""
    n = float(s.n_eff)
    if n <= 0:
        return float("nan"), float("nan")
    m = s.sum / n
    var = s.sum2 / n - m * m
    return m, float(np.sqrt(max(var, 0.0) / n))

