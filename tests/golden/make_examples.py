"""Packages the reference's four published example runs as fixtures.

The reference ships four example inputs with the log of a 10 x 50 000
trajectory run of each (one OpenMP thread), whose weighted CCS is the only
end-to-end known answer it publishes:

  acau_neutral/omega_acau_neutral_0.txt:205-206        412.887 +/- 1.471
  acau_charged/omega_acau.txt:185-186                  456.060 +/- 2.332
  change_atom_type/omega_acau_phos_sigma_0.txt:209-210 373.716 +/- 1.155
  change_atom_type/omega_acau_phos_sigma_chg_0.txt:222-223  430.892 +/- 2.297

The GPU test (tests/test_gpu_examples.py) runs on a machine without the
reference checkout, so this script stores, per example, what that test needs:
the molecule and path scalars after this library's host setup (bit for bit the
reference's setup, tests/test_host_setup.py), the run settings of the input
(trajectories per integral, integrals, progress interval) and the published
weighted CCS and error, read from the log.  Run it where the checkout is:

    python tests/golden/make_examples.py   (checkout: $COSIMS_REF, else ../reference)
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cosims_b200 import abi, host  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# fixture name -> (molecule file, input file, atom-type file, log) under examples/
EXAMPLES = {
    "ex_acau_neutral": ("acau_neutral/acau.pdb", "acau_neutral/input_neutral.txt", "",
                        "acau_neutral/omega_acau_neutral_0.txt"),
    "ex_acau_charged": ("acau_charged/acau.mfj", "", "", "acau_charged/omega_acau.txt"),
    "ex_phos_sigma": ("change_atom_type/acau_phos_sigma.pdb", "change_atom_type/input_neut.in",
                      "change_atom_type/atoms.dat",
                      "change_atom_type/omega_acau_phos_sigma_0.txt"),
    "ex_phos_sigma_chg": ("change_atom_type/acau_phos_sigma_chg.mfj",
                          "change_atom_type/input_chg.in", "change_atom_type/atoms.dat",
                          "change_atom_type/omega_acau_phos_sigma_chg_0.txt"),
}


def published(log_path: str) -> tuple:
    """(weighted CCS mean, weighted error, line of the mean) from a log."""
    lines = open(log_path).read().splitlines()
    for i, ln in enumerate(lines):
        m = re.match(r"\s*Weighted CCS Mean:\s+([0-9.]+)", ln)
        if m:
            e = re.match(r"\s*Weighted Error:\s+([0-9.]+)", lines[i + 1])
            return float(m.group(1)), float(e.group(1)), i + 1
    raise ValueError(f"no weighted mean in {log_path}")


def main() -> None:
    from oracle.refharness import REF_ROOT as ref      # $COSIMS_REF or ../reference
    if not os.path.isdir(os.path.join(ref, "examples")):
        sys.exit(f"no CoSIMS checkout at {ref}: set COSIMS_REF")
    ex = os.path.join(ref, "examples")
    for name, (mol, inp, atoms, log) in EXAMPLES.items():
        mp = os.path.join(ex, mol)
        ip = os.path.join(ex, inp) if inp else None
        ap = os.path.join(ex, atoms) if atoms else None
        cfg = host.Config(mp, ip, seed=1)
        st = host.Setup(cfg, mp, ap)
        ccs, err, line = published(os.path.join(ex, log))
        d = st.mol.to_npz_dict()
        d.update({"params_" + k: v for k, v in abi.params_to_dict(st.params).items()})
        d.update(traj=np.int64(cfg.traj), iterations=np.int64(cfg.iter),
                 print_rate=np.int64(cfg.print_rate), pub_ccs=np.float64(ccs),
                 pub_err=np.float64(err), pub_source=np.array(f"examples/{log}:{line}"))
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)
        print(f"{name}: {st.mol.n_atoms} atoms, force type {st.params.force_type}, "
              f"{cfg.iter} x {cfg.traj} trajectories, published {ccs} +/- {err}")


if __name__ == "__main__":
    main()
