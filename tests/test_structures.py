"""Multi-structure molecule files: every coordinate set of an MFJ (header
count K, records in K blocks) or PDB (MODEL .. ENDMDL blocks) gets the setup
a single-structure file of that set gets, bit for bit (rotation, boundary,
ellipsoid, clusters, path scalars)."""
import os

import numpy as np
import pytest

from cosims_b200 import abi, engine, host, synth


def _conformers(k=3, seed=5):
    base = synth.config0_molecule()
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        if i == 0:
            xyz = base.xyz.copy()
        else:
            a = rng.normal(size=3)
            a /= np.linalg.norm(a)
            t = rng.uniform(0, np.pi)
            K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
            R = np.eye(3) + np.sin(t) * K + (1 - np.cos(t)) * K @ K
            xyz = base.xyz @ R.T + rng.normal(scale=0.05, size=base.xyz.shape)
        out.append(synth.SynthMolecule(base.name, list(base.elements), xyz, base.charges,
                                       base.net_charge))
    return out


def _mfj_multi(mols, sep=True):
    first = mols[0].mfj_text().splitlines()
    head = first[:6]
    head[1] = str(len(mols))
    lines = list(head)
    for i, m in enumerate(mols):
        if i and sep:
            lines.append(str(m.n_atoms))           # a separator line between sets
        lines += m.mfj_text().splitlines()[6:]
    return "\n".join(lines) + "\n"


def _pdb_lines(m):
    out = []
    for i, (e, (x, y, z)) in enumerate(zip(m.elements, m.xyz)):
        out.append(f"{'ATOM':<6}{i + 1:5d} {e + str(i % 10):<4} {'MOL':>3} A{1:4d}    "
                   f"{x:8.3f}{y:8.3f}{z:8.3f}{1.0:6.2f}{0.0:6.2f}          {e:>2}")
    return out


def _same(a, b):
    ma, mb = a.mol, b.mol
    for k in ("xyz", "charge", "sig6", "eps24m", "eps4"):
        np.testing.assert_array_equal(getattr(ma, k), getattr(mb, k))
    for k in ("cluster_offset", "cluster_atoms", "cluster_pos", "cluster_charge",
              "cluster_dipole", "cluster_quad"):
        va, vb = getattr(ma, k, None), getattr(mb, k, None)
        assert (va is None) == (vb is None)
        if va is not None:
            np.testing.assert_array_equal(va, vb)
    np.testing.assert_array_equal(a.boundary, b.boundary)
    assert abi.params_to_dict(a.params) == abi.params_to_dict(b.params)
    for f in ("ell_a", "ell_b", "ell_c", "b_max", "mu", "radius_gyration"):
        assert getattr(a.info, f) == getattr(b.info, f)


def test_mfj_sets_equal_single_files(tmp_path):
    mols = _conformers(3)
    multi = tmp_path / "conf.mfj"
    multi.write_text(_mfj_multi(mols))
    ip = tmp_path / "conf.in"
    ip.write_text(synth.input_text("cutoff", traj_thousands=1, iterations=1))
    assert host.count_structures(str(multi)) == 3
    sets = host.setup_structures(str(multi), str(ip), seed=1, threads=4)
    assert len(sets) == 3
    for s, m in enumerate(mols):
        single = tmp_path / f"conf{s}"
        os.makedirs(single)
        mp = m.write_mfj(str(single / "conf.mfj"))
        ref = host.setup_from_files(mp, str(ip), seed=1, threads=4)
        _same(sets[s], ref)
    # the sets differ (they are different conformers)
    assert not np.array_equal(sets[0].boundary, sets[1].boundary)


def test_mfj_sets_without_separators(tmp_path):
    mols = _conformers(2, seed=9)
    a, b = tmp_path / "a.mfj", tmp_path / "b.mfj"
    a.write_text(_mfj_multi(mols, sep=True))
    b.write_text(_mfj_multi(mols, sep=False))
    for s in range(2):
        _same(host.setup_from_files(str(a), seed=2, threads=4, structure=s),
              host.setup_from_files(str(b), seed=2, threads=4, structure=s))


def test_single_structure_file_is_read_as_before(tmp_path):
    m = _conformers(1)[0]
    mp = m.write_mfj(str(tmp_path / "one.mfj"))
    assert host.count_structures(mp) == 1
    (only,) = host.setup_structures(mp, seed=3, threads=4)
    _same(only, host.setup_from_files(mp, seed=3, threads=4))


def test_pdb_models_equal_single_files(tmp_path):
    mols = _conformers(2, seed=11)
    lines = ["HEADER    CONFORMERS"]
    for i, m in enumerate(mols):
        lines += [f"MODEL     {i + 1:4d}"] + _pdb_lines(m) + ["ENDMDL"]
    lines.append("END")
    multi = tmp_path / "conf.pdb"
    multi.write_text("\n".join(lines) + "\n")
    assert host.count_structures(str(multi)) == 2
    for s, m in enumerate(mols):
        d = tmp_path / f"p{s}"
        os.makedirs(d)
        single = d / "conf.pdb"
        single.write_text("\n".join(["HEADER    CONFORMERS"] + _pdb_lines(m) + ["END"]) + "\n")
        _same(host.setup_from_files(str(multi), seed=4, threads=4, structure=s),
              host.setup_from_files(str(single), seed=4, threads=4))


def test_structure_errors(tmp_path):
    mols = _conformers(2)
    multi = tmp_path / "conf.mfj"
    multi.write_text(_mfj_multi(mols))
    with pytest.raises(engine.CosimsError):
        host.setup_from_files(str(multi), seed=1, structure=2)
    short = tmp_path / "short.mfj"
    text = _mfj_multi(mols).splitlines()
    short.write_text("\n".join(text[:-5]) + "\n")      # the last set is cut short
    with pytest.raises(engine.CosimsError):
        host.setup_from_files(str(short), seed=1, structure=1)
