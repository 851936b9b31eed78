"""Failure handling of the host side, on the CPU.

The reference's MFJ reader takes its input unchecked (molecule2::importMFJ,
molecule2.cpp:442-647): a word where a number belongs reads as 0 and "nan"
reads as NaN, and the run then integrates a wrong or non-finite molecule.
Here a corrupt record is an error with a message, a file cut short inside a
record keeps its complete records (as the reference's stream reads do) with a
warning, and the C ABI rejects non-finite molecule data before any device
work."""
import numpy as np
import pytest

from cosims_b200 import abi, engine, host, synth
from tests.common import load

HEADER = "mol\n1\n{n}\nang\ncalc\n1.0\n"


def _write(tmp_path, text, name="m.mfj"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def _records(n=6):
    mol = synth.config0_molecule()
    return mol.mfj_text().splitlines()[6:6 + n]


def test_mfj_word_in_a_coordinate_is_an_error(tmp_path):
    rec = _records()
    bad = rec[2].split()
    bad[1] = "abc"
    rec[2] = " ".join(bad)
    mp = _write(tmp_path, HEADER.format(n=len(rec)) + "\n".join(rec) + "\n")
    with pytest.raises(engine.CosimsError) as ei:
        host.setup_from_files(mp, seed=1)
    assert ei.value.status == abi.ERR_IO
    assert "not five numbers" in str(ei.value)


@pytest.mark.parametrize("token", ["nan", "inf", "-inf"])
def test_mfj_non_finite_coordinate_is_an_error(tmp_path, token):
    rec = _records()
    bad = rec[3].split()
    bad[0] = token
    rec[3] = " ".join(bad)
    mp = _write(tmp_path, HEADER.format(n=len(rec)) + "\n".join(rec) + "\n")
    with pytest.raises(engine.CosimsError) as ei:
        host.setup_from_files(mp, seed=1)
    assert ei.value.status == abi.ERR_IO
    assert "non-finite" in str(ei.value)


def test_mfj_cut_inside_a_record_keeps_the_complete_ones(tmp_path):
    rec = _records(40)
    text = HEADER.format(n=len(rec)) + "\n".join(rec[:-1]) + "\n" + \
        " ".join(rec[-1].split()[:3]) + "\n"
    mp = _write(tmp_path, text)
    ip = _write(tmp_path, synth.input_text("full"), "in.txt")
    st = host.setup_from_files(mp, ip, seed=1)
    assert st.mol.n_atoms == len(rec) - 1
    assert "complete atom records were read" in st.log


def test_mfj_without_atoms_is_an_error(tmp_path):
    mp = _write(tmp_path, HEADER.format(n=5))
    with pytest.raises(engine.CosimsError) as ei:
        host.setup_from_files(mp, seed=1)
    assert ei.value.status == abi.ERR_IO


def test_missing_molecule_file_is_an_error(tmp_path):
    with pytest.raises(engine.CosimsError) as ei:
        host.setup_from_files(str(tmp_path / "absent.mfj"), seed=1)
    assert ei.value.status == abi.ERR_IO


@pytest.mark.parametrize("field", ["xyz", "charge", "sig6", "cluster_pos"])
def test_ctx_rejects_non_finite_molecule(field):
    """cosims_ctx_create validates before it looks for a device, so this runs
    on a machine without one."""
    mol, par, _ = load("q128_t1")
    arr = getattr(mol, field).copy()
    arr.flat[1] = np.nan
    kw = {k: getattr(mol, k) for k in (
        "xyz", "charge", "sig6", "eps24m", "eps4", "cluster_offset", "cluster_atoms",
        "cluster_pos", "cluster_radius", "cluster_charge", "cluster_dipole", "cluster_quad",
        "cluster_replaced")}
    kw[field] = arr
    bad = abi.MoleculeArrays(**kw)
    with pytest.raises(engine.CosimsError) as ei:
        engine.Context(bad, par, abi.PLAIN_F64)
    assert ei.value.status == abi.ERR_INVALID
    assert "non-finite" in str(ei.value)


def test_ctx_rejects_non_finite_path_scalars():
    mol, par, _ = load("c0_t5")
    par.b_max = float("inf")
    with pytest.raises(engine.CosimsError) as ei:
        engine.Context(mol, par, abi.MIXED)
    assert ei.value.status == abi.ERR_INVALID
