"""Serving: continuous batching with admission, residency and retirement.
North-star requirement: each job's result is the same alone and in the mix.
Here it is identical, because a job's k-th round integrates trajectories
[k*R, (k+1)*R) of its own stream whatever else is running."""
import numpy as np
import pytest

from cosims_b200 import abi, engine
from tests.common import load

pytestmark = pytest.mark.gpu

NAMES = ["c0_t5", "q128_t1", "c1_t3", "q128_t4"]


def _run(jobs, round_traj=2048, target=0.02, budget=1 << 30, max_jobs=8):
    """Run jobs [(name, seed)] to completion; jobs join one per round."""
    out = {}
    with engine.Server(hbm_budget=budget, max_jobs=max_jobs, round_traj=round_traj) as srv:
        pending = list(jobs)
        ids = {}
        while pending or any(srv.poll(j).state == abi.JOB_RUNNING for j in ids):
            if pending:                           # continuous admission
                name, seed = pending[0]
                mol, par, _ = load(name)
                jid = srv.submit(mol, par, seed, target, min_traj=4096, max_traj=200000)
                if jid is not None:
                    ids[jid] = (name, seed)
                    pending.pop(0)
            srv.step()
            for jid in list(ids):
                st = srv.poll(jid)
                if st.state == abi.JOB_DONE:
                    out[ids.pop(jid)] = st
                    srv.release(jid)
    return out


def test_job_result_same_alone_and_in_the_mix():
    jobs = [(n, 40 + i) for i, n in enumerate(NAMES)]
    mixed = _run(jobs)
    for key in jobs:
        alone = _run([key])[key]
        m = mixed[key]
        assert (alone.omega, alone.se, alone.rounds, alone.sums.n) == \
            (m.omega, m.se, m.rounds, m.sums.n)
        assert m.rel_se <= 0.02 or m.sums.n >= 200000


def test_admission_by_footprint_and_slots():
    mol, par, _ = load("c1_t3")
    with engine.Server(hbm_budget=(1 << 20) * 80, max_jobs=2, round_traj=1024) as srv:
        a = srv.submit(mol, par, 1, 0.05)
        b = srv.submit(mol, par, 2, 0.05)
        assert a is not None and b is not None
        assert srv.submit(mol, par, 3, 0.05) is None          # no free slot
        srv.release(a)
        assert srv.submit(mol, par, 4, 0.05) is not None
    with engine.Server(hbm_budget=1, max_jobs=4, round_traj=16) as tiny:
        assert tiny.submit(mol, par, 1, 0.05) is None         # footprint over budget


def test_retirement_reaches_target():
    mol, par, _ = load("q128_t1")
    with engine.Server(round_traj=8192) as srv:
        j = srv.submit(mol, par, 9, 0.01, min_traj=8192)
        while srv.poll(j).state == abi.JOB_RUNNING:
            srv.step()
        st = srv.poll(j)
        assert st.rel_se <= 0.01 and st.sums.n % 8192 == 0 and st.omega > 0


def test_served_ccs_matches_plain_fp64():
    """Each retired job's Omega against the plain FP64 form run over the same
    trajectories of the job's stream (its seed, indices 0..n-1): within the
    mixed form's 0.3 % bar, at the serving configuration's 0.5 % target."""
    jobs = [(n, 70 + i) for i, n in enumerate(NAMES)]
    done = _run(jobs, round_traj=8192, target=0.005, max_jobs=4)
    for (name, seed), st in done.items():
        mol, par, _ = load(name)
        with engine.Context(mol, par, abi.PLAIN_F64) as ctx:
            s, _, _ = ctx.run_sampled(seed, 0, int(st.sums.n))
        assert s.n_hit == st.sums.n_hit
        om = s.sum / s.n_eff
        err = abs(st.omega - om) / om
        print(f"{name}: served {st.omega:.3f} ({st.sums.n} trajectories) vs plain "
              f"{om:.3f}: {100 * err:.3f} %")
        assert err <= 3e-3
