"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run where the CoSIMS reference checkout is available ($COSIMS_REF, else the
directory `reference` beside this repository):

    python tests/golden/make_golden.py

For each case it writes synthetic molecule files (cosims_b200.synth), runs
the reference's own setup and trajectory code through oracle/_ref
(libcosims_ref.so, compiled from the reference sources by oracle/Makefile),
and stores:
  - the molecule after the reference's setup (rotated coordinates, force-field
    terms, PCM clusters) and the path scalars (params_* keys);
  - forces and potentials at probe points (forceAccel::getReducedVec and
    getPotential);
  - sampled inputs and start states from monteTraj::setUpTraj;
  - per-trajectory chi / success / stepCount / energy deviation from
    diffEqSolver::verletVel for every hit;
and, for the end-to-end case, Omega as printed by the unmodified reference
binary (oracle/_ref/cosims, one thread) with the inputs its thread 0 drew.
The fixtures let the GPU tests and the oracle be checked on machines without
the reference.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cosims_b200 import abi, synth  # noqa: E402
from oracle import refharness  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def charged128() -> synth.SynthMolecule:
    """Config-0 composition with partial charges N(0, 0.3 e), net +1."""
    return synth.make_molecule("synthq128", synth.CONFIG0_COUNTS, 6.0, 1, 0.3, 77)


# name -> (molecule factory, force keyword, extra input keys, n sampled, probes)
CASES = {
    "c0_t5": (synth.config0_molecule, "cutoff", {}, 300),
    "c0_t6": (synth.config0_molecule, "full", {}, 300),
    "q128_t1": (charged128, "multipole12", {"multipole_radius": 6}, 300),
    "q128_t1_o0": (charged128, "multipole12", {"multipole_radius": 6, "multipole_order": 0}, 200),
    "q128_t2": (charged128, "multipole_full", {"multipole_radius": 6, "multipole_order": 2}, 300),
    "q128_t3": (charged128, "cutoff", {"dispersion_radius": 8}, 300),
    "q128_t4": (charged128, "full", {}, 300),
    "q128_t4_proj0": (charged128, "full", {"proj": 0}, 200),
    "c1_t3": (synth.config1_molecule, "cutoff", {}, 240),
    "c2_t1": (synth.config2_molecule, "multipole12", {}, 80),
}

SAMPLE_SEED = 7


def params_dict(p: abi.Params) -> dict:
    return {"params_" + k: np.array(v) for k, v in abi.params_to_dict(p).items()}


def probe_points(par: abi.Params, n: int, rng) -> np.ndarray:
    """Points inside the enlarged ellipsoid, at least 1.5 Angstrom from the origin."""
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = rng.uniform(0.3, 1.0, size=(n, 1))
    return u * r * np.array([par.ell_a, par.ell_b, par.ell_c])


def make_case(name: str, work: str) -> str:
    factory, force, extra, n_sample = CASES[name]
    mol = factory()
    mp, ip = synth.write_case(os.path.join(work, name), mol, force, extra=extra)
    rs = refharness.RefSetup(mp, ip, workdir=os.path.join(work, name))
    par = rs.params
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    pts = probe_points(par, 48, rng)
    acc = rs.force(pts)
    pot = rs.potential(pts)
    inputs, pos0, vel0, hit = rs.sample(n_sample, SAMPLE_SEED)
    sel = hit == 1
    chi, succ, steps, de = rs.run_list(pos0[sel], vel0[sel])
    d = dict(rs.mol.to_npz_dict())
    d.update(params_dict(par))
    d.update(
        scalars_names=np.array(list(rs.scalars.keys())),
        scalars_values=np.array(list(rs.scalars.values())),
        probe_pos=pts, probe_acc=acc, probe_pot=pot,
        inputs=inputs, start_pos=pos0, start_vel=vel0, hit=hit,
        ref_chi=chi, ref_succ=succ, ref_steps=steps, ref_de=de,
        boundary_count=np.array(rs.boundary.shape[0]),
    )
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **d)
    return path


def make_e2e(work: str, traj_k: int = 2, seed: int = 424242) -> str:
    """One integral of the unmodified reference binary on the charged 128-atom
    molecule (one thread) against the inputs its thread 0 draws."""
    mol = charged128()
    case = os.path.join(work, "e2e")
    mp, ip = synth.write_case(case, mol, "multipole12",
                              extra={"multipole_radius": 6, "threads": 1}, traj_thousands=traj_k,
                              iterations=1, name="e2e")
    rs = refharness.RefSetup(mp, ip, seed=seed, workdir=case)
    n = traj_k * 1000
    inputs, pos0, vel0, hit = rs.sample(n, seed, rand_seed=1)
    run = tempfile.mkdtemp(prefix="cosims_e2e_")
    subprocess.run([refharness.BIN_PATH, "-m", mp, "-i", ip, "-s", str(seed)], cwd=run,
                   check=True, stdout=subprocess.DEVNULL)
    logs = [f for f in os.listdir(run) if f.startswith("omega_")]
    text = open(os.path.join(run, logs[0])).read()
    om = re.search(r"Omega:\s+([0-9.]+)\s+\+/-\s+([0-9.]+)", text)
    d = dict(rs.mol.to_npz_dict())
    d.update(params_dict(rs.params))
    d.update(inputs=inputs, hit=hit, print_rate=np.array(int(rs.scalars["print_rate"])),
             omega=np.array(float(om.group(1))), omega_err=np.array(float(om.group(2))),
             n_traj=np.array(n), seed=np.array(seed))
    path = os.path.join(OUT, "e2e_q128_t1.npz")
    np.savez_compressed(path, **d)
    return path


def main(argv) -> int:
    if not refharness.available():
        print("reference checkout not found; nothing generated", file=sys.stderr)
        return 1
    names = argv[1:] or list(CASES) + ["e2e"]
    work = tempfile.mkdtemp(prefix="cosims_golden_")
    for name in names:
        path = make_e2e(work) if name == "e2e" else make_case(name, work)
        print(f"{name}: {os.path.getsize(path) / 1024:.1f} KiB -> {os.path.relpath(path, ROOT)}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
