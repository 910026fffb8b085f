"""Text outputs of SAVE_STATS_CHAN, tkebudget_chan and les_chan in the
reference's formats (for/save_stats.f:66-81,414-420,665-674,1161-1170,
for/les.f:491-503) and tkebudget_chan_les (for/save_stats.f:887-964).

The profile dictionaries come from ``Channel.save_stats()`` and
``Channel.stats_means()``.  Data rows use the reference's explicit FORMATs
(I3 then F30.20 / F20.9 / F16.9 columns).  The header lines are Fortran
list-directed writes, whose layout is compiler-specific; they are written as
space-separated values in full precision.
"""
from __future__ import annotations

import numpy as np


def _head(f, time_step: int, time: float, delta_t: float):
    f.write(f" {time_step:d} {time!r} {delta_t!r}\n")


def write_mean(path: str, st: dict, gyf: np.ndarray, time_step: int, time: float,
               delta_t: float):
    """mean.txt (for/save_stats.f:404-420): j, GYF, UME, VME on GYF, WME,
    urms, vrms, wrms, uv, uw, wv, dudy, dwdy, CP(0,0,j), shear, omega_x,
    omega_y, omega_z for j = 1..NY."""
    ny = len(gyf) - 2
    with open(path, "w") as f:
        _head(f, time_step, time, delta_t)
        f.write(f" {st['ubulk']!r}\n")
        for j in range(1, ny + 1):
            cols = [gyf[j], st["ume"][j], 0.5 * (st["vme"][j + 1] + st["vme"][j]), st["wme"][j],
                    st["urms"][j], st["vrms"][j], st["wrms"][j], st["uv"][j], st["uw"][j],
                    st["wv"][j], st["dudy"][j], st["dwdy"][j], st["cp"][j], st["shear"][j],
                    st["omega_x"][j], st["omega_y"][j], st["omega_z"][j]]
            f.write(f"{j:3d} " + "".join(f"{c:30.20f} " for c in cols) + "\n")


def write_mean_th(path: str, st: dict, gyf: np.ndarray, time_step: int, time: float,
                  delta_t: float):
    """mean_th.txt (for/save_stats.f:655-674): per scalar, j, GYF, thme,
    dthdy, thrms, thv, pe_diss for j = 1..NY."""
    ny = len(gyf) - 2
    nth = len(st["thme"])
    with open(path, "w") as f:
        _head(f, time_step, time, delta_t)
        f.write(f" {st['ubulk']!r}\n")
        for n in range(nth):
            for j in range(1, ny + 1):
                cols = [gyf[j], st["thme"][n][j], st["dthdy"][n][j], st["thrms"][n][j],
                        st["thv"][n][j], st["pe_diss"][n][j]]
                f.write(f"{j:3d} " + "".join(f"{c:30.20f} " for c in cols) + "\n")


def write_tke(path: str, st: dict, gyf: np.ndarray, time_step: int, time: float,
              delta_t: float):
    """tke.txt (for/save_stats.f:1155-1170): j, GYF, epsilon for
    j = 2..NY-1."""
    ny = len(gyf) - 2
    with open(path, "w") as f:
        _head(f, time_step, time, delta_t)
        for j in range(2, ny):
            f.write(f"{j:3d} {gyf[j]:20.9f} {st['epsilon'][j]:20.9f} \n")


def write_stats_final(path: str, means: dict, gyf: np.ndarray):
    """stats.txt of SAVE_STATS_CHAN(FINAL=.TRUE.) (for/save_stats.f:66-81):
    j, GYF, UBAR, VBAR, WBAR, then j, GYF, THBAR per scalar."""
    ny = len(gyf) - 2
    with open(path, "w") as f:
        for j in range(1, ny + 1):
            f.write(f"{j:3d},{gyf[j]:16.9f},{means['ubar'][j]:16.9f},"
                    f"{means['vbar'][j]:16.9f},{means['wbar'][j]:16.9f}\n")
        for th in means["thbar"]:
            for j in range(1, ny + 1):
                f.write(f"{j:3d},{gyf[j]:16.9f},{th[j]:16.9f}\n")


def write_mean_les(path: str, st: dict, gyf: np.ndarray, time_step: int, time: float,
                   delta_t: float):
    """mean_les.txt of les_chan (for/les.f:498-510): j, GYF, NU_T_MEAN,
    EPS_SGS1_MEAN for j = 1..NY under FORMAT (I3,' ',2(F30.20,' ')).  Four
    items against a three-item format: format reversion puts EPS_SGS1_MEAN
    on a record of its own under the repeated group."""
    ny = len(gyf) - 2
    with open(path, "w") as f:
        _head(f, time_step, time, delta_t)
        for j in range(1, ny + 1):
            f.write(f"{j:3d} {gyf[j]:30.20f} {st['nu_sgs'][j]:30.20f} \n"
                    f"{st['eps_sgs1'][j]:30.20f} \n")


def write_tke_les(path: str, epsilon_sgs: np.ndarray, gyf: np.ndarray, time_step: int,
                  time: float, delta_t: float):
    """tke_les.txt of tkebudget_chan_les (for/save_stats.f:946-960): j, GYF,
    epsilon_sgs for j = 1..NY (FORMAT I3,' ',2(F30.20,' '))."""
    ny = len(gyf) - 2

    def fw(v):
        # gfortran's F edit descriptor spells non-finite values NaN / Infinity
        if np.isnan(v):
            return "NaN".rjust(30)
        if np.isinf(v):
            return ("Infinity" if v > 0 else "-Infinity").rjust(30)
        return f"{v:30.20f}"
    with open(path, "w") as f:
        _head(f, time_step, time, delta_t)
        for j in range(1, ny + 1):
            f.write(f"{j:3d} {gyf[j]:30.20f} {fw(epsilon_sgs[j])} \n")
