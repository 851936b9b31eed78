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
