"""Wall-normal grids for the channel solver.

Restates the reference's grid pre-processor ``pre_process/create_grid_h5.m``
(lines 28-79) and the grid metrics computed on read (``for/hdf5.f:676-703``,
``for/channel.f:1646-1652``).  ``GY`` (NY+1 values, the reference's
GY(1..NY+1)) is what the solver takes; GYF/DY/DYF are derived from it exactly
as the Fortran does.
"""
from __future__ import annotations

import numpy as np

__all__ = ["create_grid", "grid_metrics", "read_ygrid_txt", "write_ygrid_txt"]


def create_grid(grid_type: int, n: int, length: float, cs: float) -> np.ndarray:
    """Return GY(1..N+1) as produced by ``create_grid_h5.m``.

    grid_type 1: tanh stretching, fine at both walls (closed channel);
    grid_type 2: cubic stretching, fine in the centre (shear layer);
    grid_type 3: as 1 but on [0, L].
    The fractional grid is then rescaled and shifted so that GYF(1) and GYF(N)
    sit where GY(1) and GY(N+1) were (create_grid_h5.m:51-71).
    """
    if n < 3:
        raise ValueError("grid needs NY >= 3")
    g = np.zeros(n + 3)
    gf = np.zeros(n + 2)
    for j in range(1, n + 2):
        x = (2.0 * (j - 1)) / n - 1.0
        if grid_type == 1:
            g[j + 1] = (length / 2.0) * np.tanh(cs * x) / np.tanh(cs)
        elif grid_type == 2:
            g[j + 1] = (length / 2.0) * (cs * x ** 3 + x) / (cs + 1)
        elif grid_type == 3:
            g[j + 1] = (length / 2.0) * np.tanh(cs * x) / np.tanh(cs) + length / 2.0
        else:
            raise ValueError("grid type must be 1, 2 or 3")
    for j in range(1, n + 1):
        gf[j + 1] = (g[j + 1] + g[j + 2]) / 2.0
    gf_lower, gf_upper = gf[2], gf[n + 1]
    g_lower, g_upper = g[2], g[n + 2]
    scale = (g_upper - g_lower) / (gf_upper - gf_lower)
    gf[2:n + 2] *= scale
    g[2:n + 3] *= scale
    shift = g_lower - gf[2]
    gf[2:n + 2] += shift
    g[2:n + 3] += shift
    return g[2:n + 3].copy()


def uniform_grid(n: int, lo: float, hi: float) -> np.ndarray:
    """GY(1..N+1) with GYF(1) = lo and GYF(N) = hi on a uniform mesh."""
    d = (hi - lo) / (n - 1)
    return lo - 0.5 * d + d * np.arange(n + 1)


def grid_metrics(gy: np.ndarray):
    """GY, GYF, DY, DYF on 0..NY+1 from GY(1..NY+1) (for/hdf5.f:676-703).

    GY(0) is left at zero as in the HDF5 read path.
    """
    gy = np.asarray(gy, dtype=np.float64)
    ny = gy.size - 1
    GY = np.zeros(ny + 2)
    GYF = np.zeros(ny + 2)
    DY = np.zeros(ny + 2)
    DYF = np.zeros(ny + 2)
    GY[1:ny + 2] = gy
    GYF[1:ny + 1] = 0.5 * (GY[1:ny + 1] + GY[2:ny + 2])
    GYF[0] = 2.0 * GYF[1] - GYF[2]
    GYF[ny + 1] = 2.0 * GYF[ny] - GYF[ny - 1]
    DY[1:ny + 2] = GYF[1:ny + 2] - GYF[0:ny + 1]
    DYF[1:ny + 1] = GY[2:ny + 2] - GY[1:ny + 1]
    DYF[ny + 1] = DYF[ny]
    return GY, GYF, DY, DYF


def read_ygrid_txt(path: str, ny: int | None = None) -> np.ndarray:
    """Read the reference's text grid (for/channel.f:1615-1633): NY, GY(1..NY+1),
    GYF(1..NY).  Returns GY(1..NY+1); raises if NY does not match."""
    with open(path) as f:
        vals = f.read().split()
    n = int(vals[0])
    if ny is not None and n != ny:
        raise ValueError(f"Error: ygrid.txt wrong dimensions (NY={ny}, file NY={n})")
    return np.array([float(v.replace("D", "E").replace("d", "e")) for v in vals[1:n + 2]])


def write_ygrid_txt(path: str, gy: np.ndarray) -> None:
    gy = np.asarray(gy, dtype=np.float64)
    ny = gy.size - 1
    gyf = 0.5 * (gy[:-1] + gy[1:])
    with open(path, "w") as f:
        f.write(f"{ny}\n")
        for v in gy:
            f.write(f"{v:.17e}\n")
        for v in gyf:
            f.write(f"{v:.17e}\n")
