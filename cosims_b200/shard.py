"""Data-parallel runs over several GPUs (one process per GPU).

Trajectories are independent, so a run shards with no collective on the data
path: rank r integrates its own counter range of the Philox stream, starting
at trajectory r * RANK_SPAN.  After the timed work the ranks exchange two
things only: the step time (max over ranks) and the CCS sums of the merged
integral (sum over ranks).  The functions take any process group, so the same
code runs over NCCL on GPUs and over gloo on CPUs (the tests).
"""
from __future__ import annotations

import math

RANK_SPAN = 10 ** 9      # trajectories reserved per rank in each stream


def first_index(rank: int, offset: int = 0) -> int:
    """First trajectory index of `rank`'s share (plus a per-step offset)."""
    return rank * RANK_SPAN + offset


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The largest `value` over the ranks (the timing rule for a whole job)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def merge_sums(sums, dist=None, device="cpu") -> dict:
    """Merged CCS of per-rank sums (objects with sum, sum2, n_eff, n, n_hit,
    n_success, max_de_pct): the totals over ranks and integrals, with
    Omega = sum / n_eff and its standard error as monteTraj::runTraj forms
    them (monteTraj.cpp:380-387)."""
    tot = [0.0] * 6
    de = 0.0
    for s in sums:
        tot[0] += s.sum
        tot[1] += s.sum2
        tot[2] += float(s.n_eff)
        tot[3] += float(s.n)
        tot[4] += float(s.n_hit)
        tot[5] += float(s.n_success)
        de = max(de, s.max_de_pct)
    if dist is not None:
        import torch
        t = torch.tensor(tot, dtype=torch.float64, device=device)
        dist.all_reduce(t)
        tot = [float(x) for x in t.cpu()]
        de = max_over_ranks(de, dist, device)
    omega = tot[0] / tot[2] if tot[2] > 0 else 0.0
    se = math.sqrt(max(tot[1] / tot[2] - omega * omega, 0.0) / tot[2]) if tot[2] > 0 else 0.0
    return {"sum": tot[0], "sum2": tot[1], "n_eff": tot[2], "n": tot[3], "n_hit": tot[4],
            "n_success": tot[5], "max_de_pct": de, "omega": omega, "se": se}
