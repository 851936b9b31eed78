"""Seeded synthetic molecules for the benchmark workloads.

A molecule is a self-avoiding random walk of 1.5 Angstrom steps inside a
confining ball of radius sqrt(5/3) * Rg_target (the radius of a uniform ball
with that radius of gyration); a new atom closer than 1.2 Angstrom to any
existing atom is rejected, and a jammed tip backtracks along the chain.
Elements are a seeded shuffle of the composition along the walk; partial
charges are N(0, sigma) shifted so that they sum to the net charge.

Output is an MFJ file the reference reads unchanged (molecule2::importMFJ,
molecule2.cpp:442-647): name, 1 coordinate set, atom count, `ang`, `calc` (or
`none` for a neutral molecule), scale 1.0, then `x y z intMass charge` lines.
Integer masses select the reference's default atom types
(molecule2.cpp:49-128): H 1, C 12, N 14, O 16, Na 23, Si 28, P 31, S 32, Fe 56.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

INT_MASS = {"H": 1, "C": 12, "N": 14, "O": 16, "Na": 23, "Si": 28, "P": 31, "S": 32, "Fe": 56}

STEP = 1.5          # Angstrom, walk step
MIN_SEP = 1.2       # Angstrom, closest allowed pair
TRIES = 24          # candidate directions per atom before backtracking


@dataclass
class SynthMolecule:
    name: str
    elements: list
    xyz: np.ndarray          # (n, 3), COM not yet removed (the reader centres it)
    charges: np.ndarray | None
    net_charge: int

    @property
    def n_atoms(self) -> int:
        return len(self.elements)

    def mfj_text(self) -> str:
        lines = [self.name, "1", str(self.n_atoms), "ang",
                 "calc" if self.charges is not None else "none", "1.0"]
        q = self.charges if self.charges is not None else np.zeros(self.n_atoms)
        for e, (x, y, z), c in zip(self.elements, self.xyz, q):
            lines.append(f"{x:14.8f} {y:14.8f} {z:14.8f} {INT_MASS[e]:4d} {c:13.8f}")
        return "\n".join(lines) + "\n"

    def write_mfj(self, path: str) -> str:
        with open(path, "w") as f:
            f.write(self.mfj_text())
        return path


def composition_counts(ratios: dict, n: int) -> dict:
    """Integer counts summing to n in the given ratios (largest remainder)."""
    tot = float(sum(ratios.values()))
    raw = {k: n * v / tot for k, v in ratios.items()}
    cnt = {k: int(math.floor(v)) for k, v in raw.items()}
    rest = n - sum(cnt.values())
    for k in sorted(raw, key=lambda k: (raw[k] - cnt[k], k), reverse=True)[:rest]:
        cnt[k] += 1
    return cnt


def random_walk(n: int, r_ball: float, rng: np.random.Generator) -> np.ndarray:
    """Self-avoiding walk of n atoms from the origin inside a ball of radius r_ball.

    Candidate directions come TRIES at a time; the first one inside the ball
    and at least MIN_SEP from every placed atom is taken, else the tip backs
    up along the chain.  Placed atoms are binned in cells of side MIN_SEP, so
    the separation test reads only the 27 cells around a candidate (the same
    distances, hence the same walk, as a test against every atom)."""
    xyz = np.zeros((n, 3))
    cap = 8                                   # atoms MIN_SEP apart: at most 8 per cell
    nc = int(math.ceil(2.0 * (r_ball + STEP) / MIN_SEP)) + 3
    grid = np.full((nc, nc, nc, cap), -1, dtype=np.int64)
    fill = np.zeros((nc, nc, nc), dtype=np.int64)
    off = (nc // 2)
    nbr = np.array([(i, j, k) for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)])

    def cell_of(p):
        return np.floor(p / MIN_SEP).astype(np.int64) + off

    c0 = cell_of(xyz[0])
    grid[c0[0], c0[1], c0[2], 0] = 0
    fill[c0[0], c0[1], c0[2]] = 1
    tip = 0
    count = 1
    guard = 0
    while count < n:
        guard += 1
        if guard > 200 * n:
            raise RuntimeError("random walk could not place all atoms")
        d = rng.normal(size=(TRIES, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        cand = xyz[tip] + STEP * d
        ok = np.linalg.norm(cand, axis=1) <= r_ball
        if ok.any():
            cells = cell_of(cand)[:, None, :] + nbr[None, :, :]          # (T, 27, 3)
            ids = grid[cells[..., 0], cells[..., 1], cells[..., 2]]      # (T, 27, cap)
            ids = ids.reshape(TRIES, -1)
            valid = ids >= 0
            diff = cand[:, None, :] - xyz[np.where(valid, ids, 0)]
            dist = np.sqrt((diff * diff).sum(axis=2))
            dist = np.where(valid, dist, np.inf)
            ok &= dist.min(axis=1) >= MIN_SEP
        idx = np.flatnonzero(ok)
        if idx.size:
            xyz[count] = cand[idx[0]]
            c = cell_of(xyz[count])
            f = fill[c[0], c[1], c[2]]
            if f >= cap:
                raise RuntimeError("cell capacity exceeded")
            grid[c[0], c[1], c[2], f] = count
            fill[c[0], c[1], c[2]] = f + 1
            tip = count
            count += 1
        else:
            tip = max(0, tip - 1 - int(rng.integers(0, 3)))   # backtrack along the chain
    return xyz


def make_molecule(name: str, counts: dict, rg_target: float, net_charge: int,
                  charge_sigma: float | None, seed: int) -> SynthMolecule:
    rng = np.random.Generator(np.random.PCG64(seed))
    elems = [e for e in sorted(counts) for _ in range(counts[e])]
    rng.shuffle(elems)
    n = len(elems)
    # A walk from the centre fills the ball unevenly; widen the ball until the
    # radius of gyration is within 4 % of the target (at most four passes).
    scale = 1.25
    for _ in range(4):
        xyz = random_walk(n, math.sqrt(5.0 / 3.0) * rg_target * scale, rng)
        c = xyz - xyz.mean(axis=0)
        rg = math.sqrt(float((c * c).sum(axis=1).mean()))
        if abs(rg - rg_target) <= 0.04 * rg_target:
            break
        scale *= rg_target / rg
    charges = None
    if charge_sigma is not None:
        q = rng.normal(0.0, charge_sigma, size=n)
        q += (net_charge - q.sum()) / n
        charges = q
    return SynthMolecule(name=name, elements=elems, xyz=xyz, charges=charges,
                         net_charge=net_charge)


# ---- the benchmark configurations --------------------------------------------

CONFIG0_COUNTS = {"C": 40, "H": 60, "N": 12, "O": 14, "P": 2}
CONFIG1_COUNTS = {"C": 160, "H": 240, "N": 48, "O": 56, "P": 8}
CONFIG2_RATIOS = {"C": 32, "H": 50, "N": 9, "O": 9, "S": 0.3}


def config0_molecule(seed: int = 0) -> SynthMolecule:
    """Neutral 128-atom molecule, Rg ~ 6 Angstrom (force type 5)."""
    return make_molecule("synth128", CONFIG0_COUNTS, 6.0, 0, None, seed)


def config1_molecule(seed: int = 1000) -> SynthMolecule:
    """512 atoms, charge +2, partial charges N(0, 0.3 e), Rg ~ 9.5 Angstrom."""
    return make_molecule("synth512", CONFIG1_COUNTS, 9.5, 2, 0.3, seed)


def config2_molecule(seed: int = 2000) -> SynthMolecule:
    """3000-atom protein-like ion, charge +10, N(0, 0.35 e), Rg ~ 15 Angstrom."""
    return make_molecule("synth3000", composition_counts(CONFIG2_RATIOS, 3000), 15.0, 10,
                         0.35, seed)


# force keys of the single-molecule configurations (input_text's names): the
# LJ cut-off for the 128- and 512-atom molecules (variants 5 and 3), the 12 A
# multipole cut-off for the 3000-atom protein (variant 1)
CONFIG_FORCE = {0: "cutoff", 1: "cutoff", 2: "multipole12"}


def config_molecule(k: int) -> SynthMolecule:
    """The molecule of single-molecule configuration k (0, 1 or 2)."""
    return {0: config0_molecule, 1: config1_molecule, 2: config2_molecule}[k]()


def config3_sizes(n_mol: int = 256, seed: int = 3000) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    n = np.exp(rng.normal(math.log(400.0), 0.9, size=n_mol))
    return np.clip(np.round(n), 50, 5000).astype(int)


def config3_charge(n_atoms: int) -> int:
    return int(min(12, round(12.0 * (n_atoms / 5000.0) ** (2.0 / 3.0))))


def config3_molecule(index: int, n_atoms: int) -> SynthMolecule:
    counts = composition_counts(CONFIG0_COUNTS, int(n_atoms))
    rg = 6.0 * (n_atoms / 128.0) ** (1.0 / 3.0)
    z = config3_charge(n_atoms)
    return make_molecule(f"synthb{index:03d}", counts, rg, z, 0.3, 3000 + index)


def input_text(force: str, traj_thousands: float = 1, iterations: int = 1,
               extra: dict | None = None, name: str | None = None) -> str:
    """Input-file text selecting the force variant the way the workloads do.

    force: 'cutoff' (multipole 0, dispersion cut-off: types 5 / 3),
           'multipole12' (multipole 1, multipole_radius 12: type 1),
           'full' (no cut-offs: types 6 / 4), 'multipole_full' (type 2).
    """
    keys = {"cutoff": {"multipole": 0, "dispersion_cutoff": 1},
            "multipole12": {"multipole": 1, "multipole_radius": 12, "dispersion_cutoff": 1},
            "full": {"multipole": 0, "dispersion_cutoff": 0},
            "multipole_full": {"multipole": 1, "dispersion_cutoff": 0}}[force]
    lines = []
    if name:
        lines.append(f"name {name}")
    lines += [f"traj {traj_thousands:g}", f"iter {iterations}"]
    for k, v in {**keys, **(extra or {})}.items():
        lines.append(f"{k} {v}")
    return "\n".join(lines) + "\n"


def write_case(dirpath: str, mol: SynthMolecule, force: str, **kw) -> tuple:
    os.makedirs(dirpath, exist_ok=True)
    mp = mol.write_mfj(os.path.join(dirpath, mol.name + ".mfj"))
    ip = os.path.join(dirpath, mol.name + "_" + force + ".in")
    with open(ip, "w") as f:
        f.write(input_text(force, **kw))
    return mp, ip
