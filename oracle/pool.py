"""The oracle over a pool of host processes.  TEST INFRASTRUCTURE ONLY.

Per-trajectory parity at the benchmark configurations' list sizes (1e4 start
states and more) needs the oracle's serial verletVel restatement on every
host core.  The pool is started with the `spawn` method, so it is safe to use
after the calling process has initialised CUDA (a forked child of a CUDA
process hangs).  Used by tests/ and by bench.py's cpu_baseline leg as the
checker; the product (cosims_b200) never imports it.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np

from cosims_b200 import abi


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _chunk(args):
    mol, pdict, pos0, vel0 = args
    from oracle import oracle
    t0 = time.perf_counter()
    out = oracle.run_list(mol, abi.params_from_dict(pdict), pos0, vel0)
    return out, time.perf_counter() - t0


def run_list(mol: abi.MoleculeArrays, par: abi.Params, pos0: np.ndarray, vel0: np.ndarray,
             workers: int = 0, chunk: int = 64) -> tuple:
    """oracle.run_list over `workers` spawned processes (0: every host core).

    Returns (records, wall seconds, summed per-chunk oracle seconds).  The
    records are in list order; each trajectory is integrated independently, so
    the split does not change a bit of them."""
    pos0 = np.ascontiguousarray(pos0, dtype=np.float64).reshape(-1, 3)
    vel0 = np.ascontiguousarray(vel0, dtype=np.float64).reshape(-1, 3)
    n = pos0.shape[0]
    if n == 0:
        return np.zeros(0, abi.TRAJ_OUT_DTYPE), 0.0, 0.0
    workers = workers or host_cores()
    pdict = abi.params_to_dict(par)
    jobs = [(mol, pdict, pos0[i:i + chunk], vel0[i:i + chunk]) for i in range(0, n, chunk)]
    t0 = time.perf_counter()
    with ProcessPoolExecutor(max_workers=min(workers, len(jobs)),
                             mp_context=mp.get_context("spawn")) as ex:
        parts = list(ex.map(_chunk, jobs))
    wall = time.perf_counter() - t0
    out = np.concatenate([p for p, _ in parts])
    return out, wall, sum(t for _, t in parts)
