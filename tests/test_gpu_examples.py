"""The reference's published example runs, reproduced on the GPU.

The reference's only end-to-end known answers are the weighted CCS of its four
example runs (10 integrals x 50 000 trajectories each, one OpenMP thread; the
logs under examples/).  tests/golden/make_examples.py packaged each example's
molecule after the host setup (bit for bit the reference's), its run settings
and the published weighted mean and error.  Here the plain FP64 form runs the
same number of integrals and trajectories, and the weighted mean is formed as
monteTraj::runTraj forms it (monteTraj.cpp:389-453): Omega_k = sum_k / n_eff_k
per integral, error sqrt((sum2/n - Omega^2) / n), inverse-variance weighted
over the integrals.  The trajectories come from the Philox stream, not the
reference's mt19937_64 stream, so the comparison is statistical: the GPU value
must lie within 3 * hypot(published error, GPU error) of the published one.
"""
import math
import os

import numpy as np
import pytest

from cosims_b200 import abi, engine
from tests.common import GOLDEN

pytestmark = pytest.mark.gpu

EXAMPLES = ["ex_acau_neutral", "ex_acau_charged", "ex_phos_sigma", "ex_phos_sigma_chg"]


def _load(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    mol = abi.MoleculeArrays.from_npz(d)
    par = abi.params_from_dict({k[len("params_"):]: d[k] for k in d if k.startswith("params_")})
    return mol, par, d


def weighted_ccs(sums):
    om = np.array([s.sum / s.n_eff for s in sums])
    err = np.array([math.sqrt((s.sum2 / s.n_eff - (s.sum / s.n_eff) ** 2) / s.n_eff)
                    for s in sums])
    w = 1.0 / err ** 2
    return float(np.sum(om * w) / np.sum(w)), float(1.0 / math.sqrt(np.sum(w)))


@pytest.mark.parametrize("name", EXAMPLES)
def test_published_example_ccs(name):
    mol, par, d = _load(name)
    n, iters, every = int(d["traj"]), int(d["iterations"]), int(d["print_rate"])
    with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
        sums = [ctx.run_sampled(seed=12345, first=k * n, n=n, update_every=every)[0]
                for k in range(iters)]
    assert all(s.n == n for s in sums)
    ccs, err = weighted_ccs(sums)
    pub, pub_err = float(d["pub_ccs"]), float(d["pub_err"])
    print(f"{name}: GPU {ccs:.3f} +/- {err:.3f}, published {pub:.3f} +/- {pub_err:.3f} "
          f"({d['pub_source']})")
    assert abs(ccs - pub) <= 3.0 * math.hypot(pub_err, err)
