"""The product's host setup (C++, include/cosims_host.h) against the reference.

The setup must reproduce the reference's molecule rotation, force-field terms,
potential-energy boundary, ellipsoid, clusters and path scalars bit for bit:
the trajectory path's parity depends on it.  Against the golden fixtures
(made by the reference) everywhere; against the live reference harness and the
published example logs where the reference checkout is present."""
import os

import numpy as np
import pytest

from cosims_b200 import abi, host, synth
from tests.common import load

from oracle.refharness import REF_ROOT as REF  # noqa: E402  ($COSIMS_REF or ../reference)
EX = os.path.join(REF, "examples")
has_ref = pytest.mark.skipif(not os.path.isdir(EX), reason="reference checkout not present")

MOL_KEYS = ("xyz", "charge", "sig6", "eps24m", "eps4", "cluster_offset", "cluster_atoms",
            "cluster_pos", "cluster_radius", "cluster_charge", "cluster_dipole", "cluster_quad",
            "cluster_replaced")


def _same(st, mol, par):
    for k in MOL_KEYS:
        np.testing.assert_array_equal(getattr(st.mol, k), getattr(mol, k), err_msg=k)
    assert abi.params_to_dict(st.params) == abi.params_to_dict(par)


GOLDEN_INPUTS = {
    "c0_t5": (synth.config0_molecule, "cutoff", {}),
    "c0_t6": (synth.config0_molecule, "full", {}),
    "q128_t1": (None, "multipole12", {"multipole_radius": 6}),
    "q128_t2": (None, "multipole_full", {"multipole_radius": 6, "multipole_order": 2}),
    "q128_t3": (None, "cutoff", {"dispersion_radius": 8}),
    "q128_t4_proj0": (None, "full", {"proj": 0}),
    "c1_t3": (synth.config1_molecule, "cutoff", {}),
}


@pytest.mark.parametrize("name", list(GOLDEN_INPUTS))
def test_setup_matches_golden(name, tmp_path):
    from tests.golden.make_golden import charged128
    factory, force, extra = GOLDEN_INPUTS[name]
    mol = (factory or charged128)()
    mp, ip = synth.write_case(str(tmp_path), mol, force, extra=extra)
    st = host.setup_from_files(mp, ip, seed=1)
    gm, gp, d = load(name)
    _same(st, gm, gp)
    assert st.boundary.shape[0] == int(d["boundary_count"])


def test_setup_thread_count_does_not_change_result(tmp_path):
    mp, ip = synth.write_case(str(tmp_path), synth.config1_molecule(), "cutoff")
    a = host.setup_from_files(mp, ip, seed=1, threads=1)
    b = host.setup_from_files(mp, ip, seed=1, threads=7)
    np.testing.assert_array_equal(a.boundary, b.boundary)
    assert abi.params_to_dict(a.params) == abi.params_to_dict(b.params)


@has_ref
@pytest.mark.parametrize("case", [
    ("acau_charged/acau.mfj", "", ""),
    ("acau_neutral/acau.pdb", "acau_neutral/input_neutral.txt", ""),
    ("change_atom_type/acau_phos_sigma.pdb", "change_atom_type/input_neut.in",
     "change_atom_type/atoms.dat"),
    ("change_atom_type/acau_phos_sigma_chg.mfj", "change_atom_type/input_chg.in",
     "change_atom_type/atoms.dat"),
])
def test_setup_matches_reference_examples(case):
    from oracle import refharness
    mol, inp, atoms = (os.path.join(EX, c) if c else "" for c in case)
    st = host.setup_from_files(mol, inp or None, atoms or None, seed=1)
    rs = refharness.RefSetup(mol, inp, atoms)
    _same(st, rs.mol, rs.params)
    np.testing.assert_array_equal(st.boundary, rs.boundary)


@has_ref
def test_published_setup_values_acau_charged():
    """Known answers printed in examples/acau_charged/omega_acau.txt:39-102."""
    st = host.setup_from_files(os.path.join(EX, "acau_charged/acau.mfj"), seed=1)
    i = st.info
    assert i.n_atoms == 252 and i.n_clusters == 18                      # :90
    assert round(i.mu, 3) == 3.996                                    # :39
    assert round(i.radius_gyration, 4) == 7.8722                       # :43
    assert [round(v, 4) for v in i.center] == [3.0444, 3.4873, 4.2035]  # :46
    assert [f"{v:.5g}" for v in (i.ell_a - i.enlarge, i.ell_b - i.enlarge,
                                  i.ell_c - i.enlarge)] == ["35.234", "35.937", "38.189"]  # :74
    assert round(i.enlarge, 2) == 1.29                                 # :85
    assert f"{i.avg_cluster_radius:.2f}" == "3.24"                     # :92
    assert f"{i.g_max:.3f}" == "40.273" and f"{i.g_min:.3f}" == "7.620"  # :98-99
    assert f"{i.pct_used:.3f}" == "98.980"                             # :102
    assert [f"{v:.4f}" for v in i.dipole] == ["2.6413", "2.0542", "-0.3638"]  # :64


@has_ref
def test_published_setup_values_acau_neutral():
    """examples/acau_neutral/omega_acau_neutral_0.txt: axes before the
    enlargement and the velocity statistics."""
    st = host.setup_from_files(os.path.join(EX, "acau_neutral/acau.pdb"),
                               os.path.join(EX, "acau_neutral/input_neutral.txt"), seed=1)
    i = st.info
    assert [f"{v:.5g}" for v in (i.ell_a - i.enlarge, i.ell_b - i.enlarge,
                                  i.ell_c - i.enlarge)] == ["22.352", "23.388", "25.164"]
    assert st.params.force_type == 5


def test_config_parsing_follows_fileparams(tmp_path):
    mp = str(tmp_path / "mol.v1.mfj")
    open(mp, "w").write("x\n")
    c = host.Config(mp)
    assert c.name == "mol" and c.traj == 50000 and c.iter == 10 and c.print_rate == 20000
    assert c.multipole == 1 and c.dispersion_cutoff == 1 and c.proj == 1 and c.dt == 0.01
    ip = str(tmp_path / "in.txt")
    open(ip, "w").write("name run\ntraj 2.5\niter 3\ncharge -2\nmultipole false\n"
                        "dispersion_cutoff 0\nbogus 1\ntraj 3\n# comment here\nincomplete\n")
    c = host.Config(mp, ip)
    assert c.name == "run_-2" and c.traj == 3000 and c.iter == 3
    assert c.charged == 1 and c.charge == -2 and c.multipole == 0 and c.dispersion_cutoff == 0
    assert c.print_rate == 600                       # traj / 5 when not given
    assert "Can not interpret option 'bogus'" in c.log
    assert "Parameter TRAJ already specified" in c.log
    assert "incomplete" in c.log
