"""The multi-rank path on CPU: two gloo ranks (127.0.0.1) run the sharding
and merging code that bench.py runs over NCCL.  Each rank integrates its own
counter range; the merged CCS must equal the CCS of all records reduced in
one place (the oracle's bookkeeping, monteTraj.cpp:380-387), and the step
time is the slower rank's."""
import math
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cosims_b200 import abi, shard
from oracle import oracle


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _records(rank: int, n: int) -> np.ndarray:
    """Per-trajectory records of rank `rank`'s share (deterministic stand-ins)."""
    rng = np.random.Generator(np.random.PCG64(shard.first_index(rank)))
    out = np.zeros(n, abi.TRAJ_OUT_DTYPE)
    out["chi"] = rng.uniform(0, math.pi, n)
    out["status"] = np.where(rng.random(n) < 0.9, abi.TRAJ_HIT | abi.TRAJ_SUCCESS, 0)
    out["de_pct"] = rng.uniform(0, 0.4, n)
    return out


def _worker(rank, world, port, n, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    par = abi.Params()
    par.ccs_const = 1.0
    s = oracle.reduce(par, _records(rank, n), 0)
    merged = shard.merge_sums([s], dist, "cpu")
    slowest = shard.max_over_ranks(10.0 + rank, dist, "cpu")
    if rank == 0:
        q.put((merged, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_merge_like_one_place():
    world, n = 2, 5000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    merged, slowest = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    par = abi.Params()
    par.ccs_const = 1.0
    # the reference's bookkeeping treats each rank's share as its own thread
    ref = [oracle.reduce(par, _records(r, n), 0) for r in range(world)]
    tot_sum = sum(s.sum for s in ref)
    tot_n = sum(s.n_eff for s in ref)
    assert merged["sum"] == pytest.approx(tot_sum, rel=1e-15)
    assert merged["n_eff"] == tot_n and merged["n"] == world * n
    assert merged["omega"] == pytest.approx(tot_sum / tot_n, rel=1e-15)
    assert slowest == 11.0
    assert shard.first_index(1) - shard.first_index(0) == shard.RANK_SPAN


def _inputs(rank: int, n: int, par) -> np.ndarray:
    """Sampled start values of rank `rank`'s trajectory range: each trajectory's
    values are a function of its global index only (as the device sampler's
    counter-based stream), drawn with the reference's distributions."""
    out = np.zeros(n, abi.TRAJ_IN_DTYPE)
    first = shard.first_index(rank)
    for i in range(n):
        rng = np.random.Generator(np.random.PCG64(first + i))
        u = rng.random(5)
        out[i] = (par.b_max * math.sqrt(u[0]), 2 * math.pi * u[1], math.acos(1 - 2 * u[2]),
                  2 * math.pi * u[3], par.g_min + (par.g_max - par.g_min) * u[4])
    return out


def _integrating_worker(rank, world, port, n, q):
    from tests.common import load
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mol, par, _ = load("c0_t5")
    out = oracle.run_inputs(mol, par, _inputs(rank, n, par))   # this rank's trajectories
    s = oracle.reduce(par, out, 0)
    merged = shard.merge_sums([s], dist, "cpu")
    if rank == 0:
        q.put(merged)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_integrating_their_ranges_merge_like_one_place():
    """Each rank integrates its own trajectory range (the oracle's verletVel
    restatement stands in for the GPU on CPU ranks); the merged CCS equals the
    same ranges integrated and reduced in one process."""
    from tests.common import load
    world, n = 2, 24
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_integrating_worker, args=(r, world, port, n, q))
             for r in range(world)]
    for p in procs:
        p.start()
    merged = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mol, par, _ = load("c0_t5")
    ref = [oracle.reduce(par, oracle.run_inputs(mol, par, _inputs(r, n, par)), 0)
           for r in range(world)]
    assert merged["sum"] == sum(s.sum for s in ref)
    assert merged["sum2"] == sum(s.sum2 for s in ref)
    assert merged["n_eff"] == sum(s.n_eff for s in ref) and merged["n"] == world * n
    assert merged["n_hit"] == sum(s.n_hit for s in ref) > 0
