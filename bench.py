#!/usr/bin/env python
"""Trajectory-method CCS throughput on B200.

Workload (one step = one CCS integral): the 512-atom synthetic ion of the
benchmark's second configuration (charge +2, partial charges N(0, 0.3 e),
exact induced-dipole electrostatics with the LJ cluster cut-off, force
variant 3), 100 000 sampled trajectories per step, He at 298 K.  The timed
form is the mixed-precision engine (FP32 pair forces, FP64 integration and
energy check); the plain FP64 form runs on the same sampled inputs to give
the CCS error of mixed against FP64 and the plain throughput.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Under torchrun every rank integrates its own
trajectories (disjoint Philox counter ranges; weak scaling) and the time is
the max over ranks.  --impl reference times the unmodified reference program
(oracle/_ref/cosims, built from the reference sources) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "trajectories/s at <=0.3% CCS err (mixed vs plain FP64); p50/p99 request latency"
UNIT = "trajectories/s"
N_TRAJ = 100_000
SEED = 20251203
# Algorithmic FP32 work per pair term, from the reference's formulas
# (forceAccel.cpp:856-884 LJ; :751-805 LJ + charge field and gradient):
# flops with FMA = 2, division and square root = 1.  A charge-field pair
# outside the LJ cut-off (variants 1-3) skips the LJ term's 14 flops.
FLOPS_LJ, FLOPS_ES, FLOPS_FAR = 22, 55, 60
FLOPS_ES_NOLJ = 41
FLOPS_POT_CHARGED, FLOPS_POT_NEUTRAL = 24, 15


def cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def workload_files(tmp: str):
    from cosims_b200 import synth
    mol = synth.config1_molecule()
    mp, ip = synth.write_case(tmp, mol, "cutoff", traj_thousands=N_TRAJ / 1000, iterations=1)
    return mol, mp, ip


# ---- clocks during the timed region ----------------------------------------------------

class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(
            ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
             "-i", str(self.device), "-lms", "200"],
            stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        time.sleep(0.3)

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9 and f[1].isdigit():
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [int(r[1]) for r in rows]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][2]),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


# ---- the reference program on the host cores ------------------------------------------

def reference_binary() -> str | None:
    p = os.path.join(ROOT, "oracle", "_ref", "cosims")
    return p if os.path.exists(p) and os.access(p, os.X_OK) else None


def run_reference(mp: str, traj: int, iters: int, threads: int, seed: int = SEED,
                  timeout: float = 1800) -> list:
    """Runs the unmodified reference program; returns per-integral trajectory
    phase times (its `Total time:` lines are cumulative, monteTraj.cpp:397)."""
    from cosims_b200 import synth
    work = tempfile.mkdtemp(prefix="cosims_refbench_")
    ip = os.path.join(work, "bench.in")
    with open(ip, "w") as f:
        f.write(synth.input_text("cutoff", traj_thousands=traj / 1000, iterations=iters,
                                 extra={"threads": threads, "print_rate": traj}, name="bench"))
    subprocess.run([reference_binary(), "-m", mp, "-i", ip, "-s", str(seed)], cwd=work,
                   check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                   timeout=timeout)
    logs = [f for f in os.listdir(work) if f.startswith("omega_")]
    text = open(os.path.join(work, logs[0])).read()
    cum = [float(x) for x in re.findall(r"Total time: ([0-9.]+);", text)]
    shutil.rmtree(work, ignore_errors=True)
    return [b - a for a, b in zip([0.0] + cum[:-1], cum)]


def reference_sample_size(target_s: float, ncores: int) -> int:
    per_core = 550.0     # trajectories/s per core of the reference on this workload
    n = int(round(per_core * ncores * target_s / 1000.0)) * 1000
    return max(1000, min(N_TRAJ, n))


def reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    if not reference_binary():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference program not built (oracle/_ref/cosims)"}))
        return
    tmp = tempfile.mkdtemp(prefix="cosims_bench_")
    _, mp, _ = workload_files(tmp)
    nc = cores()
    traj = reference_sample_size(3.0, nc)
    times = run_reference(mp, traj, args.warmup + args.steps, nc)
    timed = times[args.warmup:]
    value = traj * len(timed) / sum(timed)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * sum(timed) / len(timed), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(group_lanes=None, l2="n/a (host CPU)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nc, "kind": "reference",
                         "sample": f"{traj} trajectories per integral x {args.steps} integrals "
                                   f"(reference program, OpenMP threads = {nc})"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def config_block(group_lanes, l2) -> dict:
    return {"workload": "512-atom synthetic ion, charge +2, force variant 3 (exact "
                        "induced dipole + LJ cluster cut-off), He 298 K; one CCS integral "
                        f"of {N_TRAJ} sampled trajectories per step",
            "atoms": 512, "traj_per_step": N_TRAJ, "force_type": 3,
            "form": "mixed (FP32 pair forces, FP64 integration and energy check)",
            "group_lanes": group_lanes, "l2": l2}


# ---- our arm ------------------------------------------------------------------------------

def roofline_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
    return None


def flops_of(s, charged: bool) -> float:
    """Algorithmic flops of a work record (pair terms by kind)."""
    pot = FLOPS_POT_CHARGED if charged else FLOPS_POT_NEUTRAL
    return (FLOPS_LJ * s.pair_lj + FLOPS_ES * (s.pair_es - s.pair_es_nolj) +
            FLOPS_ES_NOLJ * s.pair_es_nolj + FLOPS_FAR * s.far_terms + pot * s.pair_pot)


def autotune(ctx, stream, torch, d_sums) -> int:
    """Lanes per trajectory for this molecule: the fastest on three integrals
    of other trajectories in one call (the timed call's steady state, where
    the integrals' long trajectories overlap the next integrals' work)."""
    from cosims_b200 import abi
    sz = abi.C.sizeof(abi.CcsSums)
    d = torch.zeros(4 * sz, dtype=torch.uint8, device="cuda")
    best, best_ms = None, 1e30
    for g in (4, 8, 16, 32):
        ctx.set_launch(group_lanes=g)
        ctx.run_integrals_device(SEED + 7, 0, N_TRAJ, 3, 0, d.data_ptr(), 0, stream)
        ms = ctx.kernel_ms()
        if ms < best_ms:
            best, best_ms = g, ms
    ctx.set_launch(group_lanes=best)
    return best


def timed_integrals(ctx, first: int, k: int, stream, torch, flush, n: int = N_TRAJ):
    """k CCS integrals of n trajectories through cosims_run_integrals_device
    (one call, device-resident records), timed on the stream with CUDA events.
    Returns (ms of the call, per-integral sums, work record)."""
    from cosims_b200 import abi
    sz = abi.C.sizeof(abi.CcsSums)
    d = torch.zeros((k + 1) * sz, dtype=torch.uint8, device="cuda")
    flush.zero_()                                   # L2 flush before the call
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    ctx.run_integrals_device(SEED, first, n, k, 0, d.data_ptr(), d.data_ptr() + k * sz, stream)
    b.record(stream)
    torch.cuda.synchronize()
    raw = d.cpu().numpy()
    sums = [abi.CcsSums.from_buffer_copy(raw[i * sz:(i + 1) * sz].tobytes()) for i in range(k)]
    work = abi.CcsSums.from_buffer_copy(raw[k * sz:(k + 1) * sz].tobytes())
    return a.elapsed_time(b), sums, work


def profile_case(args, mol, par, stream, torch) -> None:
    """A small, self-contained run for profilers (one form, few launches)."""
    from cosims_b200 import abi, engine
    prec = abi.MIXED if args.profile == "mixed" else abi.PLAIN_F64
    d_sums = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    if args.profile_max_steps:
        par = type(par).from_buffer_copy(par)
        par.max_steps = args.profile_max_steps
    with engine.Context(mol, par, prec) as ctx:
        if args.group_lanes and prec == abi.MIXED:
            ctx.set_launch(group_lanes=args.group_lanes)
        if args.profile_budget:
            ctx.set_handoff(args.profile_budget, 0)
        n = args.profile_traj
        m = max(1, args.profile_integrals)
        d_many = torch.zeros((m + 1) * abi.C.sizeof(abi.CcsSums), dtype=torch.uint8, device="cuda")
        for k in range(args.warmup + args.steps):
            if m == 1:
                ctx.run_sampled_device(SEED, k * n, n, 0, d_sums.data_ptr(), stream)
            else:               # m integrals in one launch, as the timed call runs them
                ctx.run_integrals_device(SEED, k * m * n, n, m, 0, d_many.data_ptr(), 0, stream)
            ms = ctx.kernel_ms()
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "traj": n, "launch": ctx.get_launch(),
                          "handoff": ctx.get_handoff(), "last_kernel_ms": ms}))


def parity_block(local: int) -> dict:
    """Per-trajectory parity at the configurations' list sizes, against the
    oracle on every host core (the cpu_baseline leg: the oracle is the
    checker here and its per-list time is reported).  For configurations 0
    (128-atom neutral, variant 5), 1 (512-atom +2, variant 3) and 2
    (3000-atom +10, variant 1, 12 A multipole cut-off): the first 1e4
    ellipsoid hits of the Philox stream with seed 7 through the plain FP64 and
    the mixed form on the GPU and through the oracle."""
    import numpy as np
    from cosims_b200 import abi, engine, host, synth
    from oracle import parity, pool
    n_list = 10_000
    out = {"list": f"first {n_list} ellipsoid hits of the Philox stream, seed 7",
           "bars": {"plain_frac_within_1e-6_rad": 0.99, "plain_ccs_pct": 0.1,
                    "mixed_ccs_pct_at_1e5": 0.3}}
    tmp = tempfile.mkdtemp(prefix="cosims_parity_")
    for k in (0, 1, 2):
        mp_, ip = synth.write_case(tmp, synth.config_molecule(k), synth.CONFIG_FORCE[k])
        st = host.setup_from_files(mp_, ip, seed=7, device=local)
        mol, par = st.mol, st.params
        with engine.Context(mol, par, abi.PLAIN_F64, device=local) as ctx:
            m = int(n_list * 1.4) + 64
            _, p0, v0, hit = ctx.sample_inputs(7, 0, m)
            sel = np.flatnonzero(hit == 1)[:n_list]
            p0, v0 = p0[sel], v0[sel]
            t0 = time.perf_counter()
            plain = ctx.run_list(p0, v0)
            plain_s = time.perf_counter() - t0
        with engine.Context(mol, par, abi.MIXED, device=local) as ctx:
            mixed = ctx.run_list(p0, v0)
        ref, wall, cpu_s = pool.run_list(mol, par, p0, v0)
        sp, sm = parity.compare(plain, ref), parity.compare(mixed, ref)
        out[f"config{k}"] = {
            "atoms": int(mol.n_atoms), "force_type": int(par.force_type), "n": int(len(sel)),
            "plain": {key: sp[key] for key in (
                "frac_within_tol", "outside_chaotic", "outside_other", "chaotic_in_list",
                "status_differs", "steps_differ", "max_dchi", "ccs_rel_err_pct")},
            "mixed": {key: sm[key] for key in (
                "dchi_p50", "dchi_p90", "dchi_p99", "max_dchi", "frac_within_tol",
                "outside_chaotic", "outside_other", "status_differs", "ccs_rel_err_pct")},
            "oracle": {"wall_s": round(wall, 2), "cpu_s": round(cpu_s, 2),
                       "workers": pool.host_cores(),
                       "traj_per_s_one_core": len(sel) / cpu_s if cpu_s > 0 else None},
            "gpu_plain_run_list_s": round(plain_s, 3),
        }
    shutil.rmtree(tmp, ignore_errors=True)
    return out


# ---- the batched and serving workloads (configurations 3 and 4) -------------------

def _gen_config3(args_):
    i, n = args_
    from cosims_b200 import synth
    return synth.config3_molecule(i, int(n))


def config3_library(n_mol: int, seed: int = 3000):
    """The synthetic library of the batched configuration: n_mol molecules
    with log-normal atom counts (median 400, sigma_ln 0.9, 50..5000), charge
    0..+12 growing as N^(2/3), generated in a spawn pool of host processes."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    from cosims_b200 import synth
    sizes = synth.config3_sizes(max(n_mol, 256), seed)[:n_mol]
    work = list(enumerate(sizes))
    work_sorted = sorted(work, key=lambda x: -x[1])            # big ones first
    with ProcessPoolExecutor(max_workers=max(1, min(cores(), 32)),
                             mp_context=mp.get_context("spawn")) as ex:
        mols = dict(zip([i for i, _ in work_sorted], ex.map(_gen_config3, work_sorted)))
    return [mols[i] for i in range(n_mol)], sizes


def setup_library(mols, device: int):
    """Reference setup of each molecule (boundary ray march on the GPU).
    Force variant: the LJ cut-off (3 charged / 5 neutral) up to 2000 atoms,
    the 12 A multipole cut-off (variant 1) above.  Returns the (molecule,
    params) pairs, the total seconds and each molecule's seconds."""
    from cosims_b200 import host, synth
    tmp = tempfile.mkdtemp(prefix="cosims_lib_")
    out, each = [], []
    phases = [0.0] * 6
    t0 = time.time()
    for m in mols:
        t1 = time.perf_counter()
        force = "multipole12" if m.n_atoms > 2000 else "cutoff"
        mp_, ip = synth.write_case(tmp, m, force)
        st = host.setup_from_files(mp_, ip, seed=SEED, device=device)
        out.append((st.mol, st.params))
        each.append(time.perf_counter() - t1)
        phases = [a + b for a, b in zip(phases, list(st.info.setup_ms))]
    shutil.rmtree(tmp, ignore_errors=True)
    names = ("read", "properties_rotation", "velocity_distribution", "boundary_scan_gpu",
             "ellipsoid_fit", "pcm_clusters")
    split = {k: round(v / len(mols), 3) for k, v in zip(names, phases)}
    return out, time.time() - t0, each, split


def batched_block(args, local, torch, steps: int, warmup: int, library=None) -> dict:
    """Configuration 3: 256 molecules x 2e4 trajectories in one persistent
    launch (device work queue, CUDA graph, autotuned lanes per trajectory),
    against 256 plain FP64 per-molecule launches (every molecule, timed), with
    each molecule's CCS error of batched against plain."""
    import numpy as np
    from cosims_b200 import abi, engine
    per_mol = 20000
    t0 = time.time()
    if library is None:
        mols, sizes = config3_library(args.molecules)
        gen_s = time.time() - t0
        lib_, setup_s, _, split = setup_library(mols, local)
    else:
        lib_, sizes, gen_s, setup_s, _, split = library
    ms_, pars = [m for m, _ in lib_], [p for _, p in lib_]
    k = len(ms_)
    stream = torch.cuda.current_stream()
    seeds = np.arange(k, dtype=np.uint64) + np.uint64(SEED)
    n = np.full(k, per_mol, np.int64)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    b = engine.Batch(ms_, pars, device=local)
    t1 = time.time()
    b.autotune()
    tune_s = time.time() - t1
    for w in range(warmup):
        b.run(seeds, np.full(k, w * per_mol, np.int64), n)
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    step_ms, kern_ms, sums_all, works = [], [], [], []
    for s_ in range(steps):
        flush.zero_()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sums = b.run(seeds, np.full(k, (warmup + s_) * per_mol, np.int64), n, stream)
        e.record(stream)
        torch.cuda.synchronize()
        step_ms.append(a.elapsed_time(e))
        work, kms = b.counters()
        kern_ms.append(kms)
        works.append(work)
        sums_all.append(sums)
    clk = clocks.stop()
    mean_ms = sum(step_ms) / len(step_ms)
    total = int(n.sum())
    value = total / (mean_ms / 1000.0)
    fp32_peak, _ = engine.probe_peaks(local)
    achieved = sum(flops_of(w, True) for w in works) / (sum(kern_ms) / 1000.0) / 1e12

    # plain FP64 and mixed, one launch per molecule, every molecule, on the
    # first timed step's trajectories
    first_cmp = warmup * per_mol
    ref = sums_all[0]
    plain_ms, mixed_ms, errs, ses = 0.0, 0.0, [], []
    d = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    sz = abi.C.sizeof(abi.CcsSums)
    for i in range(k):
        with engine.Context(ms_[i], pars[i], abi.PLAIN_F64, device=local) as pc:
            pc.reserve(per_mol)              # the call's buffers, outside the timed region
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            pc.run_sampled_device(int(seeds[i]), first_cmp, per_mol, 0, d.data_ptr(), stream)
            e.record(stream)
            torch.cuda.synchronize()
            plain_ms += a.elapsed_time(e)
            ps = abi.CcsSums.from_buffer_copy(d.cpu().numpy()[:sz].tobytes())
        errs.append(abs(ref[i].sum - ps.sum) / ps.sum * 100.0)
        om_p, se_p = engine.omega(ps)
        ses.append(se_p / om_p * 100.0)      # the plain integral's own statistical error
        with engine.Context(ms_[i], pars[i], abi.MIXED, device=local) as mc:
            mc.set_launch(group_lanes=b.launch(i)[0])
            mc.reserve(per_mol)
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            mc.run_sampled_device(int(seeds[i]), first_cmp, per_mol, 0, d.data_ptr(), stream)
            e.record(stream)
            torch.cuda.synchronize()
            mixed_ms += a.elapsed_time(e)
    b.close()
    plain_value = total / (plain_ms / 1000.0)
    types = sorted({int(p.force_type) for p in pars})
    errs_a = np.array(errs)
    ses_a = np.array(ses)
    worst = int(np.argmax(errs_a))
    return {
        "workload": f"batched: {k} synthetic molecules (atoms log-normal, median 400, "
                    f"sigma_ln 0.9, 50..5000; charge 0..+12 growing as N^(2/3)) x {per_mol} "
                    "trajectories, one persistent launch per step (CUDA graph)",
        "value": value, "unit": UNIT, "steps": steps, "warmup": warmup, "ms_per_step": mean_ms,
        "molecules": k, "atoms_total": int(np.sum(sizes)), "atoms_median": int(np.median(sizes)),
        "atoms_max": int(np.max(sizes)), "force_types": types, "traj_per_step": total,
        "plain_f64_per_molecule_launches": {
            "value": plain_value, "unit": UNIT, "molecules_timed": k,
            "total_ms": plain_ms},
        "mixed_per_molecule_launches": {"value": total / (mixed_ms / 1000.0), "unit": UNIT,
                                        "total_ms": mixed_ms},
        "batched_over_plain": value / plain_value,
        "batched_over_mixed_per_molecule": value / (total / (mixed_ms / 1000.0)),
        "ccs_err_pct_vs_plain": {"max": float(errs_a.max()), "mean": float(errs_a.mean()),
                                 "p90": float(np.percentile(errs_a, 90)),
                                 "within_bar": int(np.sum(errs_a <= 0.3)),
                                 "molecules": k, "bar_pct": 0.3,
                                 # the difference against the plain integral's own
                                 # standard error over the same trajectories
                                 "max_over_plain_se": float(np.max(errs_a / ses_a)),
                                 "worst": {"atoms": int(sizes[worst]),
                                           "force_type": int(pars[worst].force_type),
                                           "err_pct": float(errs_a[worst]),
                                           "plain_se_pct": float(ses_a[worst])}},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "kernel": "batch_mixed_kernel", "kernel_ms": sum(kern_ms) / len(kern_ms)},
        "host_s": {"generate": round(gen_s, 1), "setup": round(setup_s, 1),
                   "autotune": round(tune_s, 1)},
        "setup_ms_per_molecule_by_phase": split,
        "clocks": clk,
    }


def serve_stream(srv, lib_, arrivals, which, target, seed0: int, round_traj: int):
    """Feeds requests (arrival times in s, library index, target rel. SE) to
    the server and steps it until every request has retired.  Returns
    (records of done requests, wall seconds, trajectories integrated)."""
    from cosims_b200 import abi
    t0 = time.perf_counter()
    pending, live, done = 0, {}, []
    traj_done = 0
    while pending < len(arrivals) or live:
        now = time.perf_counter() - t0
        while pending < len(arrivals) and arrivals[pending] <= now:
            m, p = lib_[int(which[pending])]
            jid = srv.submit(m, p, seed0 + pending, float(target[pending]),
                             min_traj=round_traj, max_traj=400 * round_traj)
            if jid is None:
                break                                    # no room: admit later, in order
            live[jid] = pending
            pending += 1
        if not live:
            if pending < len(arrivals):
                time.sleep(max(0.0, min(0.01, arrivals[pending] - now)))
            continue
        srv.step()
        t_now = time.perf_counter() - t0
        for jid in list(live):
            stt = srv.poll(jid)
            if stt.state == abi.JOB_DONE:
                r = live.pop(jid)
                done.append({"req": r, "latency": t_now - arrivals[r], "omega": stt.omega,
                             "rel_se": stt.rel_se, "n": int(stt.sums.n),
                             "mol": int(which[r]), "target": float(target[r])})
                traj_done += stt.sums.n
                srv.release(jid)
    return done, time.perf_counter() - t0, traj_done


def serving_block(args, local, torch, library=None, duration: float | None = None) -> dict:
    """Configuration 4: CCS requests arrive as a Poisson stream; each names a
    molecule of the configuration-3 library and a target relative standard
    error (0.5 %, or 0.2 % for one request in ten).  Requests are admitted as
    slots and HBM budget free up, run in rounds with everything else in
    flight, and retire at their target.  The offered rate is 75 % of the
    capacity measured on a burst of 96 requests first (the configuration's
    50 req/s exceeds one B200's capacity for this mix).  Latency is from
    arrival to retirement; the per-molecule host setup is reported apart and
    as a second latency figure with each request's own setup time added."""
    import numpy as np
    from cosims_b200 import abi, engine
    duration = args.duration if duration is None else duration
    if library is None:
        mols, sizes = config3_library(args.molecules)
        lib_, setup_s, per_setup, _ = setup_library(mols, local)
    else:
        lib_, sizes, _, setup_s, per_setup, _ = library
    rng = np.random.Generator(np.random.PCG64(SEED))
    round_traj = 8192
    srv = engine.Server(device=local, hbm_budget=16 << 30, max_jobs=128, round_traj=round_traj)
    # warm the kernels on a few jobs
    for j in range(4):
        m, p = lib_[j]
        jid = srv.submit(m, p, 1 + j, 0.05, min_traj=round_traj, max_traj=4 * round_traj)
        while srv.poll(jid).state == abi.JOB_RUNNING:
            srv.step()
        srv.release(jid)

    def draw(nreq):
        which = rng.integers(0, len(lib_), size=nreq)
        target = np.where(rng.random(nreq) < 0.1, 0.002, 0.005)
        return which, target

    # capacity: a burst of requests all present at t = 0
    n_burst = 96
    w_b, t_b = draw(n_burst)
    done_b, wall_b, _ = serve_stream(srv, lib_, np.zeros(n_burst), w_b, t_b, 10 ** 6, round_traj)
    capacity = len(done_b) / wall_b
    rate = args.rate if args.rate > 0 else 0.75 * capacity
    n_req = int(rate * duration * 1.5) + 16
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    arrivals = arrivals[arrivals < duration]
    which, target = draw(len(arrivals))
    clocks = ClockSampler(local)
    clocks.start()
    done, wall, traj_done = serve_stream(srv, lib_, arrivals, which, target, SEED, round_traj)
    clk = clocks.stop()
    srv.close()
    lat = np.array([d_["latency"] for d_ in done])
    lat_setup = np.array([d_["latency"] + per_setup[d_["mol"]] for d_ in done])
    tgt = np.array([d_["target"] for d_ in done])
    ntraj = np.array([d_["n"] for d_ in done])
    # 5 % of the requests against the plain FP64 form on the same trajectories
    sample = done[::20]
    errs = []
    d = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    sz = abi.C.sizeof(abi.CcsSums)
    for r in sample:
        m, p = lib_[r["mol"]]
        with engine.Context(m, p, abi.PLAIN_F64, device=local) as pc:
            pc.run_sampled_device(SEED + r["req"], 0, r["n"], 0, d.data_ptr(),
                                  torch.cuda.current_stream())
            ps = abi.CcsSums.from_buffer_copy(d.cpu().numpy()[:sz].tobytes())
        om = ps.sum / ps.n_eff
        errs.append(abs(r["omega"] - om) / om * 100.0)
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None
    return {
        "workload": f"serving: Poisson arrivals for {duration:g} s at 75 % of the measured "
                    f"capacity; molecules from a {len(lib_)}-molecule configuration-3 library; "
                    "target rel. SE 0.5 % (0.2 % for 10 %)",
        "capacity_req_per_s": capacity, "offered_req_per_s": rate,
        "configured_req_per_s": 50.0,
        "requests": {"arrived": int(len(arrivals)), "completed": len(done),
                     "completed_per_s": len(done) / wall, "wall_s": wall},
        "value": traj_done / wall, "unit": UNIT,
        "latency_s": {"p50": pct(lat, 50), "p99": pct(lat, 99), "max": pct(lat, 100)},
        "latency_with_setup_s": {"p50": pct(lat_setup, 50), "p99": pct(lat_setup, 99)},
        "latency_by_target_s": {
            f"{t * 100:g}%": {"requests": int(np.sum(tgt == t)),
                              "p50": pct(lat[tgt == t], 50), "p99": pct(lat[tgt == t], 99),
                              "traj_mean": float(ntraj[tgt == t].mean()) if np.any(tgt == t)
                              else None}
            for t in (0.005, 0.002)},
        "host_setup_s_per_molecule": {"mean": setup_s / len(lib_),
                                      "max": float(np.max(per_setup))},
        "ccs_err_pct_vs_plain_f64": {"max": max(errs) if errs else None,
                                     "mean": sum(errs) / len(errs) if errs else None,
                                     "checked": len(errs), "bar_pct": 0.3},
        "round_traj": round_traj, "max_jobs": 128,
        "clocks": clk,
    }


def batched_workload(args, rank, world, local, dist, torch):
    if rank != 0:
        return
    blk = batched_block(args, local, torch, args.steps, args.warmup)
    print(json.dumps({"metric": METRIC, "n_gpus": 1, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "data": "synthetic",
                      "dtype": "fp32 pair forces / fp64 integration", **blk}))


def serving_workload(args, rank, world, local, dist, torch):
    if rank != 0:
        return
    blk = serving_block(args, local, torch)
    print(json.dumps({"metric": METRIC, "n_gpus": 1, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "data": "synthetic",
                      "dtype": "fp32 pair forces / fp64 integration", **blk}))


def molecule_workload(args, rank, world, local, dist, torch):
    """Configurations 2 and 0 as single-molecule integrals.

    protein (configuration 2): 3000-atom ion, charge +10, partial charges
    N(0, 0.35 e), the PCM far-field approximation beyond 12 A (force variant 1);
    one step = one integral of 1e6 trajectories in the mixed form; the CCS
    error against the plain FP64 form is taken on the first 1e4 of them.
    small (configuration 0): neutral 128-atom molecule (variant 5); one step =
    one integral of 1e4 trajectories in the plain FP64 form (the drop-in).
    The K timed integrals (and the W warm-up ones) are one cosims_run_integrals
    call each, as in the default line."""
    import numpy as np
    from cosims_b200 import abi, engine, host, shard, synth
    protein = args.workload == "protein"
    mol_ = synth.config2_molecule() if protein else synth.config0_molecule()
    force = "multipole12" if protein else "cutoff"
    n_traj = 1_000_000 if protein else 10_000
    form = abi.MIXED if protein else abi.PLAIN_F64
    tmp = tempfile.mkdtemp(prefix="cosims_bench_")
    mp_, ip = synth.write_case(tmp, mol_, force, traj_thousands=n_traj / 1000, iterations=1)
    st = host.setup_from_files(mp_, ip, seed=SEED, device=local)
    mol, par = st.mol, st.params
    stream = torch.cuda.current_stream()
    d = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    sz = abi.C.sizeof(abi.CcsSums)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    first0 = shard.first_index(rank)
    ctx = engine.Context(mol, par, form, device=local)
    g = None
    if form == abi.MIXED:
        best = (1e30, None)
        for lanes in (16, 32):
            ctx.set_launch(group_lanes=lanes)
            ctx.run_sampled_device(SEED + 7, 0, n_traj // 10, 0, d.data_ptr(), stream)
            best = min(best, (ctx.kernel_ms(), lanes))
        g = best[1]
        ctx.set_launch(group_lanes=g)
    # warm-up and timed integrals each through one cosims_run_integrals call;
    # the buffers of the larger call are allocated first, outside both
    ctx.reserve(max(args.warmup, args.steps) * n_traj, max(args.warmup, args.steps))
    timed_integrals(ctx, first0, args.warmup, stream, torch, flush, n_traj)
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    call_ms, sums, work = timed_integrals(ctx, first0 + args.warmup * n_traj, args.steps, stream,
                                          torch, flush, n_traj)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    kmean = ctx.kernel_ms() / args.steps if args.steps * n_traj <= (1 << 22) else call_ms / args.steps
    mean_ms = shard.max_over_ranks(call_ms / args.steps, dist, "cuda")
    value = world * n_traj / (mean_ms / 1000.0)
    achieved = flops_of(work, bool(par.charged)) / args.steps / (kmean / 1000.0) / 1e12
    fp32_peak, fp64_peak = engine.probe_peaks(local)
    peak = fp32_peak if form == abi.MIXED else fp64_peak
    merged = shard.merge_sums(sums, dist, "cuda")
    # the other form on the first 1e4 trajectories of the first timed integral
    n_cmp = 10_000
    other = engine.Context(mol, par, abi.PLAIN_F64 if form == abi.MIXED else abi.MIXED,
                           device=local)
    first_cmp = first0 + args.warmup * n_traj
    other.run_sampled_device(SEED, first_cmp, n_cmp, 0, d.data_ptr(), stream)
    so = abi.CcsSums.from_buffer_copy(d.cpu().numpy()[:sz].tobytes())
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    ctx.run_sampled_device(SEED, first_cmp, n_cmp, 0, d.data_ptr(), stream)
    e.record(stream)
    torch.cuda.synchronize()
    sf = abi.CcsSums.from_buffer_copy(d.cpu().numpy()[:sz].tobytes())
    plain_sum = so.sum if protein else sf.sum
    err = abs(sf.sum - so.sum) / plain_sum * 100.0
    other.close()
    ctx.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 pair forces / fp64 integration" if protein else "f64",
            "data": "synthetic",
            "config": {"workload": (f"3000-atom synthetic ion, charge +10, force variant "
                                    f"{par.force_type} (PCM far field beyond 12 A), mixed form, "
                                    f"{n_traj} trajectories per step") if protein else
                       (f"neutral 128-atom synthetic molecule, force variant {par.force_type}, "
                        f"plain FP64 form, {n_traj} trajectories per step"),
                       "atoms": int(mol.n_atoms), "group_lanes": g,
                       "l2": "flushed before the timed call (512 MiB write)"},
            "ccs": {"omega_A2": merged["omega"], "se_A2": merged["se"],
                    "err_pct_mixed_vs_plain": err, "compared_trajectories": n_cmp,
                    "bar_pct": 0.3},
            "roofline": {"bound": "fp32" if protein else "fp64", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "kernel": f"traj_{'mixed' if protein else 'plain'}_kernel",
                         "kernel_ms": kmean},
            "clocks": clk,
        }
        print(json.dumps(line))


def library_for_extras(args, local):
    """The configuration-3 library, generated and set up once for the batched
    and serving keys of the default line."""
    t0 = time.time()
    mols, sizes = config3_library(args.molecules)
    gen_s = time.time() - t0
    lib_, setup_s, per, split = setup_library(mols, local)
    return lib_, sizes, gen_s, setup_s, per, split


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the reference program's CPU timing and the oracle parity block")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched (configuration 3) and serving (configuration 4) keys")
    ap.add_argument("--profile", choices=["mixed", "plain"], default=None,
                    help="small case for ncu: W + K integrals of --profile-traj trajectories "
                         "of one form only, no L2 flush buffer, no sweep")
    ap.add_argument("--profile-traj", type=int, default=20000)
    ap.add_argument("--profile-budget", type=int, default=0,
                    help="hand-off step budget of the profiled run (0: the default; < 0: off)")
    ap.add_argument("--profile-max-steps", type=int, default=0,
                    help="step cap of the profiled run's trajectories (0: the default)")
    ap.add_argument("--profile-integrals", type=int, default=1,
                    help="integrals of --profile-traj trajectories per launch of the profiled run")
    ap.add_argument("--profile-config", type=int, default=1, choices=[0, 1, 2],
                    help="molecule of the profiled run: 0 the 128-atom neutral molecule, "
                         "1 the 512-atom ion (default), 2 the 3000-atom protein")
    ap.add_argument("--group-lanes", type=int, default=0)
    ap.add_argument("--workload", choices=["integral", "batched", "serving", "protein", "small"],
                    default="integral",
                    help="integral: the 512-atom ion (default line); batched: 256 molecules "
                         "in one persistent launch; serving: Poisson stream of CCS requests; "
                         "protein: the 3000-atom ion, 1e6 trajectories, mixed form; small: the "
                         "neutral 128-atom molecule, 1e4 trajectories, plain FP64 form")
    ap.add_argument("--molecules", type=int, default=256, help="batched/serving: library size")
    ap.add_argument("--rate", type=float, default=0.0,
                    help="serving: requests per second (0: 75 %% of the measured capacity)")
    ap.add_argument("--duration", type=float, default=120.0, help="serving: seconds of arrivals")
    ap.add_argument("--plain-integrals", type=int, default=3,
                    help="plain FP64 integrals timed beside the mixed line")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from cosims_b200 import abi, engine, host
    if args.workload == "batched":
        batched_workload(args, rank, world, local, dist, torch)
        return
    if args.workload == "serving":
        serving_workload(args, rank, world, local, dist, torch)
        return
    if args.workload in ("protein", "small"):
        molecule_workload(args, rank, world, local, dist, torch)
        return

    tmp = tempfile.mkdtemp(prefix="cosims_bench_")
    _, mp, ip = workload_files(tmp)
    st = host.setup_from_files(mp, ip, seed=SEED)
    mol, par = st.mol, st.params
    stream = torch.cuda.current_stream()
    if args.profile:
        if args.profile_config != 1:
            from cosims_b200 import synth
            k = args.profile_config
            mp_k, ip_k = synth.write_case(tmp, synth.config_molecule(k), synth.CONFIG_FORCE[k])
            st = host.setup_from_files(mp_k, ip_k, seed=SEED, device=local)
            mol, par = st.mol, st.params
        profile_case(args, mol, par, stream, torch)
        return
    d_sums = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    from cosims_b200 import shard
    first0 = shard.first_index(rank)          # disjoint counter range per rank
    K, W = args.steps, args.warmup

    ctx = engine.Context(mol, par, abi.MIXED, device=local)
    g = args.group_lanes or autotune(ctx, stream, torch, d_sums)
    ctx.set_launch(group_lanes=g)
    # warm-up: W integrals through the same call as the timed ones; the
    # buffers of the larger call are allocated first, outside both
    ctx.reserve(max(W, K) * N_TRAJ, max(W, K))
    timed_integrals(ctx, first0, W, stream, torch, flush)

    # timed: K integrals of N_TRAJ in one cosims_run_integrals call (integral k
    # is trajectories first + k N_TRAJ ...; the call overlaps one integral's
    # long trajectories with the next integrals' work)
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    call_ms, sums, work = timed_integrals(ctx, first0 + W * N_TRAJ, K, stream, torch, flush)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    kern_ms = ctx.kernel_ms()                 # the trajectory launch(es) of the call
    drain, end = ctx.kernel_timeline()
    ho = ctx.get_handoff()
    mean_ms = shard.max_over_ranks(call_ms / K, dist, "cuda")
    value = world * N_TRAJ / (mean_ms / 1000.0)
    one_launch = K * N_TRAJ <= (1 << 22)
    flops = flops_of(work, bool(par.charged))
    achieved = flops / ((kern_ms if one_launch else call_ms) / 1000.0) / 1e12
    fp32_peak, fp64_peak = engine.probe_peaks(local)
    tr = roofline_traffic()
    traffic = None
    if tr and tr.get("bytes_per_traj"):
        traffic = tr["bytes_per_traj"] * N_TRAJ * K

    # CCS of the timed integrals (merged over ranks)
    merged = shard.merge_sums(sums, dist, "cuda")

    # plain FP64 form on the first timed integrals (identical inputs): its
    # throughput through the same call, and the CCS error of mixed against it
    P = min(args.plain_integrals, K)
    plain = engine.Context(mol, par, abi.PLAIN_F64, device=local)
    plain.reserve(P * N_TRAJ, P)
    plain.run_integrals(SEED, first0 + W * N_TRAJ, 20000, 1)           # warm
    plain_ms, psums, pwork = timed_integrals(plain, first0 + W * N_TRAJ, P, stream, torch, flush)
    plain_value = world * N_TRAJ / (shard.max_over_ranks(plain_ms / P, dist, "cuda") / 1000.0)
    errs = [abs(sums[i].sum - psums[i].sum) / psums[i].sum * 100.0 for i in range(P)]
    pooled = abs(sum(x.sum for x in sums[:P]) - sum(x.sum for x in psums)) / \
        sum(x.sum for x in psums) * 100.0
    plain_kern = plain.kernel_ms()
    plain_achieved = flops_of(pwork, bool(par.charged)) / (plain_kern / 1000.0) / 1e12

    # end to end through the C ABI with host buffers: the start states of the
    # K timed integrals (their ellipsoid hits) in pinned host memory, through
    # one cosims_run_list call, the per-trajectory records back into pinned
    # host memory; copies inside the timed region
    def pinned(x):
        return torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
    p_all, v_all = [], []
    for k in range(K):
        _, p0, v0, hit = ctx.sample_inputs(SEED, first0 + (W + k) * N_TRAJ, N_TRAJ)
        p_all.append(p0[hit == 1])
        v_all.append(v0[hit == 1])
    p_host, v_host = pinned(np.concatenate(p_all)), pinned(np.concatenate(v_all))
    n_e2e = p_host.shape[0]
    out_pinned = torch.zeros(n_e2e * abi.TRAJ_OUT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    out_host = out_pinned.numpy().view(abi.TRAJ_OUT_DTYPE)
    ctx.run_list(p_host[:20000], v_host[:20000], stream, out=out_host[:20000])      # warm
    flush.zero_()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    ctx.run_list(p_host, v_host, stream, out=out_host)
    b.record(stream)
    torch.cuda.synchronize()
    e2e_ms = shard.max_over_ranks(a.elapsed_time(b), dist, "cuda")
    e2e_value = world * n_e2e / (e2e_ms / 1000.0)

    cpu, parity = None, None
    extras = rank == 0 and world == 1
    if extras and not args.no_cpu_baseline and reference_binary():
        nc = cores()
        traj = reference_sample_size(10.0, nc)
        t = run_reference(mp, traj, 1, nc)
        cpu = {"value": traj / t[0], "unit": UNIT, "cores": nc, "kind": "reference",
               "sample": f"one integral of {traj} trajectories of the same molecule and "
                         f"input (reference program, OpenMP threads = {nc})"}
    if extras and not args.no_cpu_baseline:
        parity = parity_block(local)
    batched = serving = None
    if extras and not args.no_extras:
        library = library_for_extras(args, local)
        batched = batched_block(args, local, torch, 5, 3, library)
        serving = serving_block(args, local, torch, library)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": mean_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 pair forces / fp64 integration", "data": "synthetic",
            "config": config_block(g, f"the timed call's per-trajectory buffers (start states, "
                                      f"hits, work order, records, about 120 B x {K * N_TRAJ}) "
                                      "exceed L2; also flushed before the call (512 MiB write)"),
            "ccs": {"omega_A2": merged["omega"], "se_A2": merged["se"],
                    "err_pct_mixed_vs_plain": {"per_integral_max": max(errs),
                                               "pooled": pooled, "integrals": P},
                    "bar_pct": 0.3},
            "plain_f64": {"value": plain_value, "ms_per_step": plain_ms / P, "integrals": P,
                          "roofline": {"bound": "fp64", "achieved": plain_achieved,
                                       "peak": fp64_peak, "frac": plain_achieved / fp64_peak,
                                       "kernel": "traj_plain_kernel", "kernel_ms": plain_kern}},
            "mixed_over_plain": value / plain_value,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": traffic,
                         "kernel": f"traj_mixed_kernel<{par.force_type}>",
                         "kernel_ms": kern_ms, "launches": 1 if one_launch else None,
                         "peak_source": "measured in this run: FP32 FMA chains "
                                        "(cosims_probe_peaks); the driver's peaks file holds "
                                        "only HBM and bf16 tensor figures",
                         "fp64_peak": fp64_peak},
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(48 * n_e2e / K),
                    "d2h_bytes_per_step": int(24 * n_e2e / K),
                    "path": "cosims_run_list: pinned host start states of the K timed "
                            "integrals' ellipsoid hits -> device -> pinned host per-trajectory "
                            "records, one call (misses, resolved by the sampler, are not "
                            "counted)"},
            # sampler, 3 x work order, trajectory kernel, work counters, 2 x reduce per integral
            "gpu_launches": 6 + 2 * K,
            "clocks": clk,
            "tail": {"queue_drained_ms": round(drain, 2), "kernel_end_ms": round(end, 2),
                     "handoff": {"step_budget": ho[0], "wide_lanes": ho[1], "parked": ho[2]}},
            "batched": batched,
            "serving": serving,
        }
        print(json.dumps(line))
    ctx.close()
    plain.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
