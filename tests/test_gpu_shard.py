"""The multi-rank path with the engine: two processes share the one GPU, each a
gloo rank (127.0.0.1) that integrates its own counter range of the Philox
stream through the engine, as bench.py's ranks do over NCCL.  Their kernels
never wait on one another; the ranks meet only on the host, to merge the sums
after the work.  The merged CCS must equal the same two ranges integrated in
one process (monteTraj.cpp:380-387 for the merged bookkeeping)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cosims_b200 import abi, engine, shard
from tests.common import load

pytestmark = pytest.mark.gpu

SEED, N = 11, 4000


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, precision, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        mol, par, _ = load(name)
        with engine.Context(mol, par, precision, device=0) as ctx:
            s, _, _ = ctx.run_sampled(SEED, shard.first_index(rank), N)
        merged = shard.merge_sums([s], dist, "cpu")
        slowest = shard.max_over_ranks(float(rank), dist, "cpu")
        if rank == 0:
            q.put((merged, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,precision", [("c1_t3", abi.MIXED), ("c0_t5", abi.PLAIN_F64)])
def test_two_ranks_on_the_engine_merge_like_one_process(name, precision):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, precision, q))
             for r in range(world)]
    for p in procs:
        p.start()
    merged, slowest = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    mol, par, _ = load(name)
    with engine.Context(mol, par, precision, device=0) as c:
        ref = [c.run_sampled(SEED, shard.first_index(r), N)[0] for r in range(world)]
    # the same kernels on the same ranges: the sums are bitwise the one-process ones
    assert merged["sum"] == ref[0].sum + ref[1].sum
    assert merged["sum2"] == ref[0].sum2 + ref[1].sum2
    assert merged["n_eff"] == ref[0].n_eff + ref[1].n_eff
    assert merged["n_hit"] == ref[0].n_hit + ref[1].n_hit > 0
    assert merged["n"] == world * N
    assert merged["omega"] == (ref[0].sum + ref[1].sum) / (ref[0].n_eff + ref[1].n_eff)
    assert slowest == 1.0
