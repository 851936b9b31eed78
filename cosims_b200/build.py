"""Builds the CUDA library in-tree (cosims_b200/_lib/libcosims_cuda.so).

Runs make in cosims_b200/csrc: nvcc -gencode arch=compute_100a,code=sm_100a.
nvcc cross-compiles, so this works on a machine without a GPU.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8, verbose: bool = False) -> str:
    csrc = os.path.join(HERE, "csrc")
    cmd = ["make", "-C", csrc, f"-j{jobs}"]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return os.path.join(HERE, "_lib", "libcosims_cuda.so")


if __name__ == "__main__":
    print(build(verbose=True))
