"""Shared helpers for the tests: golden fixtures and small cases."""
from __future__ import annotations

import functools
import os

import numpy as np

from cosims_b200 import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASES = ["c0_t5", "c0_t6", "q128_t1", "q128_t1_o0", "q128_t2", "q128_t3", "q128_t4",
         "q128_t4_proj0", "c1_t3", "c2_t1"]


@functools.lru_cache(maxsize=None)
def _load(name: str):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    mol = abi.MoleculeArrays.from_npz(d)
    par = abi.params_from_dict({k[len("params_"):]: d[k] for k in d if k.startswith("params_")})
    return mol, par, d


def load(name: str):
    """(MoleculeArrays, Params, dict of arrays) of a golden fixture.  The
    Params are a fresh copy: a test that changes a setting (max_steps, say)
    leaves the fixture as it was for the tests after it."""
    mol, par, d = _load(name)
    return mol, type(par).from_buffer_copy(par), d


def hits(d):
    sel = d["hit"] == 1
    return d["start_pos"][sel], d["start_vel"][sel]


@functools.lru_cache(maxsize=None)
def config_setup(k: int, device: int | None = None):
    """(MoleculeArrays, Params) of benchmark configuration k (0: 128-atom
    neutral, 1: 512-atom +2 ion, 2: 3000-atom +10 protein with the 12 A
    multipole cut-off) after the reference setup.  `device` runs the boundary
    ray march on that GPU (bit for bit the host's)."""
    import tempfile
    from cosims_b200 import host, synth
    tmp = tempfile.mkdtemp(prefix="cosims_cfg_")
    mp, ip = synth.write_case(tmp, synth.config_molecule(k), synth.CONFIG_FORCE[k])
    st = host.setup_from_files(mp, ip, seed=7, device=device)
    return st.mol, st.params
