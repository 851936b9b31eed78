"""Python bindings of the oracle (oracle/liboracle.so).  TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
checker.  The product (cosims_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

from cosims_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_LOCK = threading.Lock()


def build() -> str:
    """Compile liboracle.so with gcc (seconds); returns its path."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return os.path.join(HERE, "liboracle.so")


def lib():
    global _LIB
    with _LOCK:
        if _LIB is None:
            path = os.path.join(HERE, "liboracle.so")
            src = os.path.join(HERE, "cosims_oracle.c")
            if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
                build()
            L = C.CDLL(path)
            P = C.POINTER
            L.oracle_force.argtypes = [P(abi.Molecule), P(abi.Params), C.c_void_p, C.c_void_p]
            L.oracle_potential.argtypes = [P(abi.Molecule), P(abi.Params), C.c_void_p]
            L.oracle_potential.restype = C.c_double
            L.oracle_run_list.argtypes = [P(abi.Molecule), P(abi.Params), C.c_int64,
                                          C.c_void_p, C.c_void_p, C.c_void_p]
            L.oracle_run_inputs.argtypes = [P(abi.Molecule), P(abi.Params), C.c_int64,
                                            C.c_void_p, C.c_void_p]
            L.oracle_verlet_trace.argtypes = [P(abi.Molecule), P(abi.Params), C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                              C.c_void_p]
            L.oracle_start_state.argtypes = [P(abi.Params), C.c_void_p, C.c_void_p, C.c_void_p]
            L.oracle_start_state.restype = C.c_int
            L.oracle_reduce.argtypes = [P(abi.Params), C.c_int64, C.c_void_p, C.c_int64,
                                        P(abi.CcsSums)]
            L.oracle_omega.argtypes = [P(abi.CcsSums), P(C.c_double), P(C.c_double)]
            _LIB = L
    return _LIB


def force(mol: abi.MoleculeArrays, par: abi.Params, pos: np.ndarray) -> np.ndarray:
    L, m = lib(), mol.view()
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    out = np.zeros_like(pos)
    for i in range(pos.shape[0]):
        L.oracle_force(C.byref(m), C.byref(par), abi.vptr(pos[i]), abi.vptr(out[i]))
    return out


def potential(mol: abi.MoleculeArrays, par: abi.Params, pos: np.ndarray) -> np.ndarray:
    L, m = lib(), mol.view()
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    return np.array([L.oracle_potential(C.byref(m), C.byref(par), abi.vptr(pos[i]))
                     for i in range(pos.shape[0])])


def run_list(mol: abi.MoleculeArrays, par: abi.Params, pos0: np.ndarray,
             vel0: np.ndarray) -> np.ndarray:
    L, m = lib(), mol.view()
    pos0 = np.ascontiguousarray(pos0, dtype=np.float64).reshape(-1, 3)
    vel0 = np.ascontiguousarray(vel0, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(pos0.shape[0], dtype=abi.TRAJ_OUT_DTYPE)
    L.oracle_run_list(C.byref(m), C.byref(par), pos0.shape[0], abi.vptr(pos0),
                      abi.vptr(vel0), abi.vptr(out))
    return out


def trace(mol: abi.MoleculeArrays, par: abi.Params, pos0: np.ndarray, vel0: np.ndarray,
          max_frames: int):
    """verletVel with a per-step record: (frames [n, max_frames, 6], steps [n], outs)."""
    L, m = lib(), mol.view()
    pos0 = np.ascontiguousarray(pos0, dtype=np.float64).reshape(-1, 3)
    vel0 = np.ascontiguousarray(vel0, dtype=np.float64).reshape(-1, 3)
    n = pos0.shape[0]
    frames = np.zeros((n, max(max_frames, 1), 6))
    steps = np.zeros(n, np.int32)
    out = np.zeros(n, dtype=abi.TRAJ_OUT_DTYPE)
    for i in range(n):
        L.oracle_verlet_trace(C.byref(m), C.byref(par), abi.vptr(pos0[i]), abi.vptr(vel0[i]),
                              abi.vptr(out[i:i + 1]), abi.vptr(frames[i]), int(max_frames),
                              abi.vptr(steps[i:i + 1]))
    return frames[:, :max_frames], steps, out


def run_inputs(mol: abi.MoleculeArrays, par: abi.Params, inputs: np.ndarray) -> np.ndarray:
    L, m = lib(), mol.view()
    inputs = np.ascontiguousarray(inputs, dtype=abi.TRAJ_IN_DTYPE)
    out = np.zeros(inputs.shape[0], dtype=abi.TRAJ_OUT_DTYPE)
    L.oracle_run_inputs(C.byref(m), C.byref(par), inputs.shape[0], abi.vptr(inputs),
                        abi.vptr(out))
    return out


def start_states(par: abi.Params, inputs: np.ndarray):
    L = lib()
    inputs = np.ascontiguousarray(inputs, dtype=abi.TRAJ_IN_DTYPE)
    n = inputs.shape[0]
    pos0, vel0 = np.zeros((n, 3)), np.zeros((n, 3))
    hit = np.zeros(n, np.int32)
    for i in range(n):
        hit[i] = L.oracle_start_state(C.byref(par), abi.vptr(inputs[i:i + 1]),
                                      abi.vptr(pos0[i]), abi.vptr(vel0[i]))
    return pos0, vel0, hit


def reduce(par: abi.Params, out: np.ndarray, update_every: int) -> abi.CcsSums:
    L = lib()
    out = np.ascontiguousarray(out, dtype=abi.TRAJ_OUT_DTYPE)
    s = abi.CcsSums()
    L.oracle_reduce(C.byref(par), out.shape[0], abi.vptr(out), int(update_every), C.byref(s))
    return s


def omega(s: abi.CcsSums):
    L = lib()
    o, e = C.c_double(), C.c_double()
    L.oracle_omega(C.byref(s), C.byref(o), C.byref(e))
    return o.value, e.value
