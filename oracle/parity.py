"""Per-trajectory parity statistics of an engine run against the oracle on the
same fixed list of start states.  TEST INFRASTRUCTURE ONLY (tests/ and
bench.py's cpu_baseline leg).

The quantities are the ones the drop-in bar is stated in:

- the fraction of trajectories whose scattering angle chi agrees with the
  oracle's within 1e-6 rad (bar: >= 99 %), with the ones outside counted and
  classed as chaotic (an energy or orbit retry, or more than 2048 steps: the
  multi-collision trajectories in which a last-bit difference grows) or not;
- the CCS of the list, sum of 2 sin^2(chi / 2) = 1 - cos(chi) over the list
  times the CCS constant (monteTraj.cpp:471-475), as a relative error against
  the oracle's (bar: 0.1 % for the plain form, 0.3 % for the mixed form);
- |d chi| percentiles, which describe the mixed form's FP32 pair forces.
"""
from __future__ import annotations

import numpy as np

from cosims_b200 import abi

CHAOTIC_STEPS = 2048


def ccs_sum(out: np.ndarray) -> float:
    """Sum of 1 - cos(chi) over the records (2 sin^2(chi/2), no cancellation)."""
    s = np.sin(0.5 * np.abs(out["chi"]))
    return float(np.sum(2.0 * s * s))


def chaotic(out: np.ndarray) -> np.ndarray:
    st = out["status"].astype(np.int64)
    retries = ((st >> abi.TRAJ_ETRIES_SHIFT) & 0xff) + ((st >> abi.TRAJ_OTRIES_SHIFT) & 0xff)
    return (retries > 0) | (out["steps"] > CHAOTIC_STEPS)


def compare(got: np.ndarray, ref: np.ndarray, tol: float = 1e-6) -> dict:
    """Statistics of `got` against the oracle's records `ref` (same list)."""
    assert got.shape == ref.shape
    n = int(got.shape[0])
    if n == 0:
        return {"n": 0}
    d = np.abs(got["chi"] - ref["chi"])
    outside = d > tol
    ch = chaotic(ref) | chaotic(got)
    s_got, s_ref = ccs_sum(got), ccs_sum(ref)
    q = np.percentile(d, [50, 90, 99])
    return {
        "n": n,
        "within_tol": int(np.sum(~outside)),
        "frac_within_tol": float(np.mean(~outside)),
        "tol_rad": tol,
        "outside_chaotic": int(np.sum(outside & ch)),
        "outside_other": int(np.sum(outside & ~ch)),
        "chaotic_in_list": int(np.sum(ch)),
        "status_differs": int(np.sum(got["status"] != ref["status"])),
        "steps_differ": int(np.sum(got["steps"] != ref["steps"])),
        "max_dchi": float(d.max()),
        "dchi_p50": float(q[0]), "dchi_p90": float(q[1]), "dchi_p99": float(q[2]),
        "ccs_rel_err_pct": 100.0 * abs(s_got - s_ref) / s_ref if s_ref > 0 else 0.0,
    }
