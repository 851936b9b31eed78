"""The oracle restatement against the reference's own outputs (golden fixtures).

The fixtures were produced by tests/golden/make_golden.py from the reference
sources (oracle/_ref).  Everything here is bit-exact: the oracle keeps the
reference's IEEE operation order, so forces, potentials, start states and
whole trajectories must agree exactly.
"""
import numpy as np
import pytest

from cosims_b200 import abi
from oracle import oracle
from tests.common import CASES, hits, load


@pytest.mark.parametrize("name", CASES)
def test_forces_and_potential_bit_exact(name):
    mol, par, d = load(name)
    np.testing.assert_array_equal(oracle.force(mol, par, d["probe_pos"]), d["probe_acc"])
    np.testing.assert_array_equal(oracle.potential(mol, par, d["probe_pos"]), d["probe_pot"])


@pytest.mark.parametrize("name", CASES)
def test_start_states_bit_exact(name):
    mol, par, d = load(name)
    pos0, vel0, hit = oracle.start_states(par, d["inputs"])
    np.testing.assert_array_equal(hit, d["hit"])
    sel = hit == 1
    np.testing.assert_array_equal(pos0[sel], d["start_pos"][sel])
    np.testing.assert_array_equal(vel0[sel], d["start_vel"][sel])


@pytest.mark.parametrize("name", [c for c in CASES if c != "c2_t1"])
def test_trajectories_bit_exact(name):
    mol, par, d = load(name)
    p0, v0 = hits(d)
    out = oracle.run_list(mol, par, p0, v0)
    np.testing.assert_array_equal(out["chi"], d["ref_chi"])
    np.testing.assert_array_equal((out["status"] & abi.TRAJ_SUCCESS) > 0, d["ref_succ"] == 1)
    np.testing.assert_array_equal(out["steps"], d["ref_steps"])
    np.testing.assert_array_equal(out["de_pct"], d["ref_de"])


def test_trajectories_bit_exact_large():
    """3000-atom protein-like ion, force type 1 (multipole far field, 12 A)."""
    mol, par, d = load("c2_t1")
    p0, v0 = hits(d)
    k = 24
    out = oracle.run_list(mol, par, p0[:k], v0[:k])
    np.testing.assert_array_equal(out["chi"], d["ref_chi"][:k])
    np.testing.assert_array_equal(out["steps"], d["ref_steps"][:k])


def test_end_to_end_omega_matches_reference_binary():
    """One integral of the unmodified reference program (one thread, 2000
    trajectories): the oracle, fed the inputs the program's thread 0 drew,
    reproduces the Omega it printed (two decimals, monteTraj.cpp:392-394)."""
    import os
    from tests.common import GOLDEN
    d = dict(np.load(os.path.join(GOLDEN, "e2e_q128_t1.npz")))
    mol = abi.MoleculeArrays.from_npz(d)
    par = abi.params_from_dict({k[7:]: d[k] for k in d if k.startswith("params_")})
    out = oracle.run_inputs(mol, par, d["inputs"])
    np.testing.assert_array_equal((out["status"] & abi.TRAJ_HIT) > 0, d["hit"] == 1)
    s = oracle.reduce(par, out, int(d["print_rate"]))
    om, err = oracle.omega(s)
    assert abs(om - float(d["omega"])) <= 0.005 + 1e-12
    assert abs(err - float(d["omega_err"])) <= 0.005 + 1e-12


def test_reduce_bookkeeping_quirks():
    """monteTraj's one-thread counting: a miss keeps the previous success flag,
    and only failures after the last progress update are subtracted."""
    par = abi.Params()
    par.ccs_const = 2.0
    S, F, M = (abi.TRAJ_HIT | abi.TRAJ_SUCCESS), abi.TRAJ_HIT, 0
    st = [S, F, M, M, S, M, F, M]
    out = np.zeros(len(st), abi.TRAJ_OUT_DTYPE)
    out["status"] = st
    out["chi"] = [0.5, np.pi / 2, 0, 0, 1.0, 0, np.pi / 2, 0]
    # update every 3: counter reset after trajectories 3 and 6; window = [6, 8)
    s = oracle.reduce(par, out, 3)
    assert s.n == 8 and s.n_hit == 4 and s.n_success == 2
    assert s.n_eff == 8 - 2            # traj 6 fails, traj 7 (miss) inherits failure
    s = oracle.reduce(par, out, 4)     # window empty: 8 % 4 == 0
    assert s.n_eff == 8
    s = oracle.reduce(par, out, 0)     # never reset: all effective failures
    # effective: S F F F S S F F -> 5 failures
    assert s.n_eff == 3
    expect = sum(2.0 * (1 - np.cos(c)) for c in out["chi"])
    assert abs(s.sum - expect) < 1e-12
