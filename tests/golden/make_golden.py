"""Regenerates the committed golden fixtures from the reference checkout.

Run in a container that has the reference mounted (its location is passed
with --ref).  Fixtures written here:
  kh_grid_y.txt   the 66 GY values stored in the reference's KH_test/grid.h5
                  (dataset /grids/y), extracted as the contiguous little-endian
                  float64 run in the file, with the byte offset recorded
  kh_input/       verbatim copies of KH_test/input.dat, input_chan.dat,
                  input_per.dat, grid_def, grid_def.all, grid_mpi (input-format
                  fixtures for the parsers)
"""
import argparse
import os
import shutil

import numpy as np


def extract_grid(path, n):
    b = open(path, "rb").read()
    for off in range(0, len(b) - n * 8 + 1):
        a = np.frombuffer(b[off:off + n * 8], dtype="<f8")
        if np.all(np.isfinite(a)) and np.all(np.diff(a) > 0) and np.all(np.abs(a) < 1e3):
            return off, a.copy()
    raise RuntimeError("grid run not found")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the reference's diablo_2.0 directory")
    args = ap.parse_args()
    here = os.path.dirname(os.path.abspath(__file__))
    kh = os.path.join(args.ref, "KH_test")
    off, gy = extract_grid(os.path.join(kh, "grid.h5"), 66)
    with open(os.path.join(here, "kh_grid_y.txt"), "w") as f:
        f.write(f"# KH_test/grid.h5 /grids/y, float64 LE at byte offset {off}, {gy.size} values\n")
        for v in gy:
            f.write(f"{v:.17e}\n")
    dst = os.path.join(here, "kh_input")
    os.makedirs(dst, exist_ok=True)
    for name in ("input.dat", "input_chan.dat", "input_per.dat", "grid_def", "grid_def.all",
                 "grid_mpi"):
        shutil.copy(os.path.join(kh, name), os.path.join(dst, name))


if __name__ == "__main__":
    main()
