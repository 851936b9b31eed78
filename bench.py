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
# flops with FMA = 2, division and square root = 1.
FLOPS_LJ, FLOPS_ES, FLOPS_FAR = 22, 55, 60
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


def autotune(ctx, stream, torch, d_sums) -> int:
    """Lanes per trajectory for this molecule: the fastest over two integrals
    of other trajectories (one integral's time varies with its longest few)."""
    best, best_ms = None, 1e30
    for g in (4, 8, 16, 32):
        ctx.set_launch(group_lanes=g)
        ms = 0.0
        for k in range(2):
            ctx.run_sampled_device(SEED + 7, k * N_TRAJ, N_TRAJ, 0, d_sums.data_ptr(), stream)
            ms += ctx.kernel_ms()
        if ms < best_ms:
            best, best_ms = g, ms
    ctx.set_launch(group_lanes=best)
    return best


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
        for k in range(args.warmup + args.steps):
            ctx.run_sampled_device(SEED, k * n, n, 0, d_sums.data_ptr(), stream)
            ms = ctx.kernel_ms()
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "traj": n, "launch": ctx.get_launch(),
                          "handoff": ctx.get_handoff(), "last_kernel_ms": ms}))


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
    the 12 A multipole cut-off (variant 1) above."""
    from cosims_b200 import host, synth
    tmp = tempfile.mkdtemp(prefix="cosims_lib_")
    out = []
    t0 = time.time()
    for m in mols:
        force = "multipole12" if m.n_atoms > 2000 else "cutoff"
        mp_, ip = synth.write_case(tmp, m, force)
        st = host.setup_from_files(mp_, ip, seed=SEED, device=device)
        out.append((st.mol, st.params))
    shutil.rmtree(tmp, ignore_errors=True)
    return out, time.time() - t0


def batched_workload(args, rank, world, local, dist, torch):
    """Configuration 3: 256 molecules x 2e4 trajectories in one persistent
    launch (device work queue, CUDA graph, autotuned lanes per trajectory),
    against per-molecule plain FP64 launches timed on a stratified subset."""
    import numpy as np
    from cosims_b200 import abi, engine
    per_mol = 20000
    t0 = time.time()
    mols, sizes = config3_library(args.molecules)
    gen_s = time.time() - t0
    lib_, setup_s = setup_library(mols, local)
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
    from cosims_b200 import shard
    first0 = shard.first_index(rank)
    for w in range(args.warmup):
        b.run(seeds, np.full(k, first0 + w * per_mol, np.int64), n)
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, kern_ms, sums_all = [], [], []
    for s_ in range(args.steps):
        flush.zero_()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sums = b.run(seeds, np.full(k, first0 + (args.warmup + s_) * per_mol, np.int64), n,
                     stream)
        e.record(stream)
        torch.cuda.synchronize()
        step_ms.append(a.elapsed_time(e))
        work, kms = b.counters()
        kern_ms.append(kms)
        sums_all.append(sums)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    mean_ms = shard.max_over_ranks(sum(step_ms) / len(step_ms), dist, "cuda")
    total = int(n.sum())
    value = world * total / (mean_ms / 1000.0)
    flops = FLOPS_LJ * work.pair_lj + FLOPS_ES * work.pair_es + FLOPS_FAR * work.far_terms + \
        FLOPS_POT_CHARGED * work.pair_pot
    fp32_peak, _ = engine.probe_peaks(local)
    achieved = flops / (kern_ms[-1] / 1000.0) / 1e12

    # plain FP64, one launch per molecule, on every 16th molecule by size
    order = np.argsort(sizes)
    subset = [int(i) for i in order[::max(1, k // 16)]]
    first_cmp = first0 + args.warmup * per_mol
    ref = sums_all[0]
    plain_ms, errs, mixed_ms = 0.0, [], 0.0
    d = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    sz = abi.C.sizeof(abi.CcsSums)
    for i in subset:
        with engine.Context(ms_[i], pars[i], abi.PLAIN_F64, device=local) as pc:
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            pc.run_sampled_device(int(seeds[i]), first_cmp, per_mol, 0, d.data_ptr(), stream)
            e.record(stream)
            torch.cuda.synchronize()
            plain_ms += a.elapsed_time(e)
            ps = abi.CcsSums.from_buffer_copy(d.cpu().numpy()[:sz].tobytes())
        errs.append(abs(ref[i].sum - ps.sum) / ps.sum * 100.0)
        with engine.Context(ms_[i], pars[i], abi.MIXED, device=local) as mc:
            mc.set_launch(group_lanes=b.launch(i)[0])
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            mc.run_sampled_device(int(seeds[i]), first_cmp, per_mol, 0, d.data_ptr(), stream)
            e.record(stream)
            torch.cuda.synchronize()
            mixed_ms += a.elapsed_time(e)
    scale = k / len(subset)
    plain_value = total / (plain_ms * scale / 1000.0)
    # the subset is stratified by size: scale its time to the 256 molecules
    b.close()
    if rank == 0:
        types = sorted({int(p.force_type) for p in pars})
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 pair forces / fp64 integration", "data": "synthetic",
            "config": {"workload": f"batched: {k} synthetic molecules (atoms log-normal, median "
                                   f"400, 50..5000; charge 0..+12) x {per_mol} trajectories, "
                                   "one persistent launch per step (CUDA graph)",
                       "molecules": k, "atoms_total": int(sizes.sum()),
                       "atoms_median": int(np.median(sizes)), "atoms_max": int(sizes.max()),
                       "force_types": types, "traj_per_step": total,
                       "l2": "flushed between steps (512 MiB write)"},
            "ccs": {"err_pct_batched_mixed_vs_plain": {"max": max(errs),
                                                        "mean": sum(errs) / len(errs),
                                                        "molecules": len(subset)},
                    "bar_pct": 0.3},
            "plain_f64_per_molecule_launches": {
                "value": plain_value, "unit": UNIT,
                "estimate": f"{len(subset)} molecules (every {k // len(subset)}th by size) "
                            f"x {per_mol} trajectories, time scaled by {scale:g}"},
            "mixed_per_molecule_launches": {"value": total / (mixed_ms * scale / 1000.0),
                                            "unit": UNIT},
            "batched_over_plain": value / world / plain_value,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": None,
                         "kernel": "batch_mixed_kernel", "kernel_ms": kern_ms[-1]},
            "host_s": {"generate": round(gen_s, 1), "setup": round(setup_s, 1),
                       "autotune": round(tune_s, 1)},
            "gpu_launches": 3 * args.steps,   # sample, trajectories, reduce (one graph)
            "clocks": clk,
        }
        print(json.dumps(line))


def serving_workload(args, rank, world, local, dist, torch):
    """Configuration 4: CCS requests arrive as a Poisson stream; each names a
    molecule of the configuration-3 library and a target relative standard
    error (0.5 %, or 0.2 % for one request in ten).  Requests are admitted as
    slots and HBM budget free up, run in rounds through the persistent kernel
    with everything else in flight, and retire at their target.  Latency is
    from arrival to retirement; the molecules' host setup is done beforehand
    and reported apart."""
    import numpy as np
    from cosims_b200 import abi, engine
    if rank != 0:
        return
    mols, sizes = config3_library(args.molecules)
    lib_, setup_s = setup_library(mols, local)
    rng = np.random.Generator(np.random.PCG64(SEED))
    n_req = int(args.rate * args.duration * 1.5) + 16
    gaps = rng.exponential(1.0 / args.rate, size=n_req)
    arrivals = np.cumsum(gaps)
    arrivals = arrivals[arrivals < args.duration]
    which = rng.integers(0, len(lib_), size=len(arrivals))
    target = np.where(rng.random(len(arrivals)) < 0.1, 0.002, 0.005)
    round_traj = 8192
    srv = engine.Server(device=local, hbm_budget=16 << 30, max_jobs=128, round_traj=round_traj)
    # warm the kernels and the tuning on a few jobs
    for j in range(4):
        m, p = lib_[j]
        jid = srv.submit(m, p, 1 + j, 0.05, min_traj=round_traj, max_traj=4 * round_traj)
        while srv.poll(jid).state == abi.JOB_RUNNING:
            srv.step()
        srv.release(jid)
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    pending, live, done = 0, {}, []
    traj_done = 0
    while pending < len(arrivals) or live:
        now = time.perf_counter() - t0
        while pending < len(arrivals) and arrivals[pending] <= now:
            m, p = lib_[int(which[pending])]
            jid = srv.submit(m, p, SEED + pending, float(target[pending]), min_traj=round_traj,
                             max_traj=400 * round_traj)
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
                done.append((r, t_now - arrivals[r], stt.omega, stt.rel_se, stt.sums.n,
                             int(which[r]), float(target[r])))
                traj_done += stt.sums.n
                srv.release(jid)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    lat = np.array([d_[1] for d_ in done])
    # CCS of a small sample against the plain FP64 form on the same trajectories
    sample = done[:: max(1, len(done) // 3)][:3]
    errs = []
    d = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    sz = abi.C.sizeof(abi.CcsSums)
    for (r, _, om, _, ntr, mi, _) in sample:
        m, p = lib_[mi]
        with engine.Context(m, p, abi.PLAIN_F64, device=local) as pc:
            pc.run_sampled_device(SEED + r, 0, int(ntr), 0, d.data_ptr(),
                                  torch.cuda.current_stream())
            ps = abi.CcsSums.from_buffer_copy(d.cpu().numpy()[:sz].tobytes())
        errs.append(abs(om - ps.sum / ps.n_eff) / (ps.sum / ps.n_eff) * 100.0)
    srv.close()
    line = {
        "metric": METRIC, "value": traj_done / wall, "unit": UNIT, "n_gpus": 1,
        "steps": len(done), "warmup": 4, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 pair forces / fp64 integration", "data": "synthetic",
        "config": {"workload": f"serving: Poisson arrivals at {args.rate:g} req/s for "
                               f"{args.duration:g} s; molecules from a {len(lib_)}-molecule "
                               "configuration-3 library; target rel. SE 0.5 % (0.2 % for 10 %)",
                   "round_traj": round_traj, "max_jobs": 128},
        "requests": {"arrived": int(len(arrivals)), "completed": len(done),
                     "admitted": int(pending), "per_s": len(done) / wall,
                     "wall_s": wall},
        "latency_s": {"p50": float(np.percentile(lat, 50)) if len(lat) else None,
                      "p99": float(np.percentile(lat, 99)) if len(lat) else None,
                      "max": float(lat.max()) if len(lat) else None},
        "ccs": {"err_pct_vs_plain_f64": errs, "sample": len(errs), "bar_pct": 0.3},
        "host_setup_s_per_molecule": setup_s / len(lib_),
        "clocks": clk,
    }
    print(json.dumps(line))


def molecule_workload(args, rank, world, local, dist, torch):
    """Configurations 2 and 0 as single-molecule integrals.

    protein (configuration 2): 3000-atom ion, charge +10, partial charges
    N(0, 0.35 e), the PCM far-field approximation beyond 12 A (force variant 1);
    one step = one integral of 1e6 trajectories in the mixed form; the CCS
    error against the plain FP64 form is taken on the first 1e4 of them.
    small (configuration 0): neutral 128-atom molecule (variant 5); one step =
    one integral of 1e4 trajectories in the plain FP64 form (the drop-in)."""
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
    step_sums = torch.zeros((args.steps, 128), dtype=torch.uint8, device="cuda")
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
    for w in range(args.warmup):
        ctx.run_sampled_device(SEED, first0 + w * n_traj, n_traj, 0, d.data_ptr(), stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms, kern = [], []
    for k in range(args.steps):
        flush.zero_()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.run_sampled_device(SEED, first0 + (args.warmup + k) * n_traj, n_traj, 0,
                               step_sums[k].data_ptr(), stream)
        e.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(e))
        kern.append(ctx.kernel_ms())
    if dist:
        dist.barrier()
    clk = clocks.stop()
    mean_ms = shard.max_over_ranks(sum(ms) / len(ms), dist, "cuda")
    value = world * n_traj / (mean_ms / 1000.0)
    raw = step_sums.cpu().numpy()
    sums = [abi.CcsSums.from_buffer_copy(raw[k, :sz].tobytes()) for k in range(args.steps)]
    pot_flops = FLOPS_POT_CHARGED if par.charged else FLOPS_POT_NEUTRAL
    flops = [FLOPS_LJ * x.pair_lj + FLOPS_ES * x.pair_es + FLOPS_FAR * x.far_terms +
             pot_flops * x.pair_pot for x in sums]
    kmean = sum(kern) / len(kern)
    achieved = sum(flops) / len(flops) / (kmean / 1000.0) / 1e12
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
                       "l2": "flushed between steps (512 MiB write)"},
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", choices=["mixed", "plain"], default=None,
                    help="small case for ncu: W + K integrals of --profile-traj trajectories "
                         "of one form only, no L2 flush buffer, no sweep")
    ap.add_argument("--profile-traj", type=int, default=20000)
    ap.add_argument("--profile-budget", type=int, default=0,
                    help="hand-off step budget of the profiled run (0: the default; < 0: off)")
    ap.add_argument("--profile-max-steps", type=int, default=0,
                    help="step cap of the profiled run's trajectories (0: the default)")
    ap.add_argument("--group-lanes", type=int, default=0)
    ap.add_argument("--workload", choices=["integral", "batched", "serving", "protein", "small"],
                    default="integral",
                    help="integral: the 512-atom ion (default line); batched: 256 molecules "
                         "in one persistent launch; serving: Poisson stream of CCS requests; "
                         "protein: the 3000-atom ion, 1e6 trajectories, mixed form; small: the "
                         "neutral 128-atom molecule, 1e4 trajectories, plain FP64 form")
    ap.add_argument("--molecules", type=int, default=256, help="batched/serving: library size")
    ap.add_argument("--rate", type=float, default=50.0, help="serving: requests per second")
    ap.add_argument("--duration", type=float, default=60.0, help="serving: seconds of arrivals")
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
        profile_case(args, mol, par, stream, torch)
        return
    d_sums = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    step_sums = torch.zeros((args.steps, 128), dtype=torch.uint8, device="cuda")
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    from cosims_b200 import shard
    first0 = shard.first_index(rank)          # disjoint counter range per rank

    ctx = engine.Context(mol, par, abi.MIXED, device=local)
    g = autotune(ctx, stream, torch, d_sums)
    for w in range(args.warmup):
        ctx.run_sampled_device(SEED, first0 + w * N_TRAJ, N_TRAJ, 0, d_sums.data_ptr(), stream)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    kern_ms = []
    sz = abi.C.sizeof(abi.CcsSums)
    tails, parked = [], []
    for k in range(args.steps):
        flush.zero_()                                   # L2 flush between steps
        ev[k][0].record(stream)
        ctx.run_sampled_device(SEED, first0 + (args.warmup + k) * N_TRAJ, N_TRAJ, 0,
                               step_sums[k].data_ptr(), stream)
        ev[k][1].record(stream)
        kern_ms.append(ctx.kernel_ms())
        drain, end = ctx.kernel_timeline()
        tails.append((drain, end))
        parked.append(ctx.get_handoff()[2])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    mean_ms = shard.max_over_ranks(sum(step_ms) / len(step_ms), dist, "cuda")
    value = world * N_TRAJ / (mean_ms / 1000.0)

    # work counters of the timed steps -> algorithmic flops of the trajectory kernel
    raw = step_sums.cpu().numpy()
    sums = [abi.CcsSums.from_buffer_copy(raw[k, :sz].tobytes()) for k in range(args.steps)]
    pot_flops = FLOPS_POT_CHARGED if par.charged else FLOPS_POT_NEUTRAL
    flops = [FLOPS_LJ * s.pair_lj + FLOPS_ES * s.pair_es + FLOPS_FAR * s.far_terms +
             pot_flops * s.pair_pot for s in sums]
    kmean = sum(kern_ms) / len(kern_ms)
    achieved = sum(flops) / len(flops) / (kmean / 1000.0) / 1e12
    fp32_peak, fp64_peak = engine.probe_peaks(local)
    tr = roofline_traffic()
    traffic = None
    if tr and tr.get("bytes_per_traj"):
        traffic = tr["bytes_per_traj"] * N_TRAJ

    # CCS of the timed integrals (merged over ranks)
    merged = shard.merge_sums(sums, dist, "cuda")
    omega, omega_se = merged["omega"], merged["se"]

    # plain FP64 form on identical inputs: throughput and the CCS error of mixed
    plain = engine.Context(mol, par, abi.PLAIN_F64, device=local)
    first_cmp = first0 + args.warmup * N_TRAJ
    plain.run_sampled_device(SEED, first_cmp, 20000, 0, d_sums.data_ptr(), stream)  # warm
    flush.zero_()
    pe = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    pe[0].record(stream)
    plain.run_sampled_device(SEED, first_cmp, N_TRAJ, 0, d_sums.data_ptr(), stream)
    pe[1].record(stream)
    torch.cuda.synchronize()
    plain_ms = pe[0].elapsed_time(pe[1])
    ps = abi.CcsSums.from_buffer_copy(d_sums.cpu().numpy()[:sz].tobytes())
    ms0 = sums[0]
    ccs_err = abs(ms0.sum - ps.sum) / ps.sum * 100.0

    # end to end through the C ABI with host buffers: the start states of the
    # same K timed integrals (their ellipsoid hits) in pinned host memory, the
    # per-trajectory records back into pinned host memory, copies inside the
    # timed region
    def pinned(x):
        return torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
    lists = []
    for k in range(args.steps):
        _, p0, v0, hit = ctx.sample_inputs(SEED, first0 + (args.warmup + k) * N_TRAJ, N_TRAJ)
        lists.append((pinned(p0[hit == 1]), pinned(v0[hit == 1])))
    n_max = max(p.shape[0] for p, _ in lists)
    out_pinned = torch.zeros(n_max * abi.TRAJ_OUT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    out_host = out_pinned.numpy().view(abi.TRAJ_OUT_DTYPE)
    ctx.run_list(lists[0][0], lists[0][1], stream, out=out_host[:lists[0][0].shape[0]])
    e2e_ms, n_list = [], []
    for k in range(args.steps):
        p0, v0 = lists[k]
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.run_list(p0, v0, stream, out=out_host[:p0.shape[0]])
        b.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(a.elapsed_time(b))
        n_list.append(p0.shape[0])
    e2e_mean = shard.max_over_ranks(sum(e2e_ms) / len(e2e_ms), dist, "cuda")
    n_e2e = sum(n_list) / len(n_list)
    e2e_value = world * n_e2e / (e2e_mean / 1000.0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and reference_binary():
        nc = cores()
        traj = reference_sample_size(10.0, nc)
        t = run_reference(mp, traj, 1, nc)
        cpu = {"value": traj / t[0], "unit": UNIT, "cores": nc, "kind": "reference",
               "sample": f"one integral of {traj} trajectories of the same molecule and "
                         f"input (reference program, OpenMP threads = {nc})"}

    ho = ctx.get_handoff()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mean_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 pair forces / fp64 integration", "data": "synthetic",
            "config": config_block(g, "flushed between steps (512 MiB write)"),
            "ccs": {"omega_A2": omega, "se_A2": omega_se,
                    "err_pct_mixed_vs_plain": ccs_err, "bar_pct": 0.3},
            "plain_f64": {"value": N_TRAJ / (plain_ms / 1000.0), "ms_per_step": plain_ms},
            "mixed_over_plain": value / world / (N_TRAJ / (plain_ms / 1000.0)),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": traffic,
                         "kernel": "traj_mixed_kernel<3>",
                         "kernel_ms": kmean,
                         "peak_source": "measured in this run: FP32 FMA chains "
                                        "(cosims_probe_peaks); the driver's peaks file holds "
                                        "only HBM and bf16 tensor figures",
                         "fp64_peak": fp64_peak},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(48 * n_e2e),
                    "d2h_bytes_per_step": int(24 * n_e2e),
                    "path": "cosims_run_list: pinned host start states of each timed "
                            "integral's ellipsoid hits -> device -> pinned host per-trajectory "
                            "records (misses, resolved by the sampler, are not counted)"},
            "gpu_launches": 7 * args.steps,   # sample, 3 x work order, trajectories, 2 x reduce
            "clocks": clk,
            "tail": {"queue_drained_ms": [round(a, 2) for a, _ in tails],
                     "kernel_end_ms": [round(b, 2) for _, b in tails],
                     "handoff": {"step_budget": ho[0], "wide_lanes": ho[1],
                                 "parked_per_step": parked}},
        }
        print(json.dumps(line))
    ctx.close()
    plain.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
