"""The command-line driver (cosims_gpu): the reference program's command
line, input file and omega_<name>.txt lines.  The GPU test runs both forms on
a synthetic 128-atom molecule and, where the reference program was built
(oracle/_ref/cosims), checks the CCS against it within the joint statistical
error (the two programs draw different random trajectories)."""
import math
import os
import re
import subprocess

import pytest

from cosims_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cosims_b200", "_lib", "cosims_gpu")
REF = os.path.join(ROOT, "oracle", "_ref", "cosims")

OMEGA = re.compile(r" Omega:\s+([0-9.]+) \+/- ([0-9.]+)\s*\(\s*([0-9.]+) %\)")


def _case(tmp_path, traj_k=2, iters=2):
    m = synth.config0_molecule()
    return synth.write_case(str(tmp_path), m, "cutoff", traj_thousands=traj_k, iterations=iters)


def test_cli_rejects_bad_arguments():
    if not os.path.exists(CLI):
        pytest.skip("command-line driver not built")
    r = subprocess.run([CLI, "-x", "1"], capture_output=True, text=True, timeout=60)
    assert "Check command line arguments" in r.stdout
    r = subprocess.run([CLI, "-i", "in.txt"], capture_output=True, text=True, timeout=60)
    assert "No molecule file" in r.stdout


def _parse(path):
    text = open(path).read()
    om = [(float(a), float(b)) for a, b, _ in OMEGA.findall(text)]
    w = re.search(r"Weighted CCS Mean:\s+([0-9.]+)", text)
    werr = re.search(r"Weighted Error:\s+([0-9.]+)", text)
    return text, om, float(w.group(1)), float(werr.group(1))


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_cli_omega_file(tmp_path, form):
    mp, ip = _case(tmp_path)
    r = subprocess.run([CLI, "-m", mp, "-i", ip, "-s", "11", "-p", form], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = [f for f in os.listdir(tmp_path) if f.startswith("omega_")]
    assert len(out) == 1
    text, om, wmean, werr = _parse(os.path.join(tmp_path, out[0]))
    assert len(om) == 2 and "Mean Cross-section" in text and "Max Energy Deviation" in text
    assert all(o > 0 and 0 < e < 0.1 * o for o, e in om)
    if os.path.exists(REF):
        subprocess.run([REF, "-m", mp, "-i", ip, "-s", "11"], cwd=str(tmp_path), check=True,
                       capture_output=True, timeout=1200)
        ref = [f for f in os.listdir(tmp_path) if f.startswith("omega_")]
        # the reference rewrites the same file name: compare its weighted mean
        _, rom, rmean, rerr = _parse(os.path.join(tmp_path, ref[0]))
        assert abs(rmean - wmean) < 4 * math.hypot(rerr, werr)


@pytest.mark.gpu
def test_cli_sets_and_dumps(tmp_path):
    """A two-set MFJ: each set's integrals and summary, the average over sets,
    and the debugging dumps (print_mol, print_data, print_traj) in the
    reference's line formats; the data lines are the successful trajectories
    of the same integrals run through the engine."""
    import numpy as np
    from cosims_b200 import abi, engine, host
    from tests.test_structures import _conformers, _mfj_multi
    mols = _conformers(2, seed=21)
    mp = tmp_path / "conf.mfj"
    mp.write_text(_mfj_multi(mols))
    ip = tmp_path / "conf.in"
    ip.write_text(synth.input_text("cutoff", traj_thousands=0.5, iterations=2,
                                   extra={"print_mol": 1, "print_data": 1, "print_traj": 1}))
    r = subprocess.run([CLI, "-m", str(mp), "-i", str(ip), "-s", "5"], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    omega = [f for f in os.listdir(tmp_path) if f.startswith("omega_")]
    text = open(tmp_path / omega[0]).read()
    assert "Coordinate set 1 / 2" in text and "Coordinate set 2 / 2" in text
    assert "Average CCS:" in text and text.count("Weighted CCS Mean:") == 2
    name = omega[0][len("omega_"):-len(".txt")]
    for s in (1, 2):
        tag = f"{name}_set{s}"
        mol_xyz = (tmp_path / f"outMol_{tag}.xyz").read_text().splitlines()
        assert mol_xyz[1] == "Rotated Molecule " and len(mol_xyz) == 2 + mols[0].n_atoms
        # data lines: the successful hits of both integrals, in index order
        st = host.setup_from_files(str(mp), str(ip), seed=5, structure=s - 1)
        want = []
        with engine.Context(st.mol, st.params, abi.PLAIN_F64) as ctx:
            for k in range(2):
                _, ins, outs = ctx.run_sampled(5, k * 500, 500, want_records=True)
                ins2, p0, v0, hit = ctx.sample_inputs(5, k * 500, 500)
                for i in np.nonzero((outs["status"] & abi.TRAJ_SUCCESS) > 0)[0]:
                    want.append("%8.3g  %8.3g  %8.3g  %8.3g  %8.3g  %8.3g  %8i  %8.3g  %8.3g  "
                                "%8.3g  %8.3g  %8.3g  %8.3g " % (
                                    ins["phi"][i], ins["theta"][i], ins["gamma"][i], ins["g"][i],
                                    ins["b"][i], outs["chi"][i], outs["steps"][i], *p0[i],
                                    *v0[i]))
        got = (tmp_path / f"data_{tag}.txt").read_text().splitlines()
        assert got == want
        frames = (tmp_path / f"xyz_{tag}.xyz").read_text().splitlines()
        assert len(frames) % 3 == 0 and len(frames) > 0
        assert frames[0] == "1" and frames[1] == "no comments available "
        assert frames[2].startswith("He     ") and len(frames[2].split()) == 7
