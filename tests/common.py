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
