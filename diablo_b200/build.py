"""Build the in-tree CUDA library (sm_100a) with the Makefile in csrc/."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdiablo_b200.so")


def build_library(jobs: int = 8, quiet: bool = True) -> str:
    r = subprocess.run(["make", "-C", CSRC, f"-j{jobs}"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("CUDA build failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    if not quiet:
        print(r.stdout)
    return LIB
