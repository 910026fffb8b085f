"""Seeded initial conditions (host side).

The reference builds its initial fields in ``CREATE_FLOW_CHAN`` /
``CREATE_TH_CHAN`` / ``CREATE_FLOW_PER`` (``for/set_ics.f``) with the
compiler's intrinsic RNG, which cannot be reproduced.  These generators keep
the reference's structure (profile on GYF planes 0..NY, noise of amplitude
KICK on every plane 0..NY+1 in physical space, scalar on planes 1..NY) and
draw the noise from numpy's PCG64 with an explicit seed, so the same input is
fed to the oracle and to the GPU path.  The spectral projection
(FFT, APPLY_BC_VEL, REM_DIV_CHAN, APPLY_BC_VEL) is done by the solver.
"""
from __future__ import annotations

import numpy as np

from .grid import grid_metrics
from .params import Params

__all__ = ["kh_shear_layer", "channel_laminar", "periodic_spectrum", "ensemble_kh_params",
           "to_spectral_chan", "kh_state"]


def _noise(rng, shape, kind, amp):
    if kind == "uniform":
        # KICK*(RNUM-0.5), for/set_ics.f:82-93
        return amp * (rng.random(shape) - 0.5)
    return amp * rng.standard_normal(shape)


def kh_shear_layer(p: Params, gy: np.ndarray, seed: int = 1, kick: float = 1e-3):
    """IC_TYPE 3 (for/set_ics.f:63-73,237-245): U1 = TH = tanh(GYF)."""
    _, GYF, _, _ = grid_metrics(gy)
    shp = p.phys_shape()
    rng = np.random.Generator(np.random.PCG64(seed))
    u1 = np.zeros(shp)
    u1[: p.ny + 1] = np.tanh(GYF[: p.ny + 1])[:, None, None]
    u2 = np.zeros(shp)
    u3 = np.zeros(shp)
    n = _noise(rng, (3,) + shp, "uniform", kick)
    u1 += n[0]
    u2 += n[1]
    u3 += n[2]
    th = np.zeros((max(p.n_th, 1),) + shp)
    for k in range(p.n_th):
        th[k, 1: p.ny + 1] = np.tanh(GYF[1: p.ny + 1])[:, None, None]
    return u1, u2, u3, th[: p.n_th]


def channel_laminar(p: Params, gy: np.ndarray, seed: int = 2, amp_frac: float = 0.1):
    """IC_TYPE 0 (for/set_ics.f:26-36): U1 = 3/2 UBULK0 (1 - GYF^2) plus a seeded
    Gaussian perturbation of amp_frac*UBULK0 on all three components (made
    divergence-free by REM_DIV_CHAN in the solver)."""
    _, GYF, _, _ = grid_metrics(gy)
    shp = p.phys_shape()
    rng = np.random.Generator(np.random.PCG64(seed))
    u1 = np.zeros(shp)
    u1[: p.ny + 1] = ((3.0 / 2.0) * p.ubulk0 * (1.0 - GYF[: p.ny + 1] ** 2))[:, None, None]
    n = _noise(rng, (3,) + shp, "gauss", amp_frac * p.ubulk0)
    u1 = u1 + n[0]
    u2 = n[1].copy()
    u3 = n[2].copy()
    th = np.zeros((p.n_th,) + shp)
    for k in range(p.n_th):
        th[k, 1: p.ny + 1] = np.tanh(GYF[1: p.ny + 1])[:, None, None]
    return u1, u2, u3, th


def periodic_spectrum(p: Params, seed: int = 3, k0: float = 4.0, u_rms: float = 1.0):
    """Random-phase solenoidal velocity with E(k) ~ k^4 exp(-2 (k/k0)^2) on the
    retained modes (a new CREATE_FLOW_PER variant; the reference only has a
    Taylor-Green vortex and an ideal vortex, for/set_ics.f:278-319).

    Returns spectral (CU1, CU2, CU3) in the retained layout [TNKY+1][TNKZ+1][NKX+1]
    with the kx = 0 plane Hermitian-symmetric so the field is real.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    nkx, nky, nkz = p.nkx, p.nky, p.nkz
    ky = np.concatenate([np.arange(nky + 1), -np.arange(nky, 0, -1)]) * (2 * np.pi / p.ly)
    kz = np.concatenate([np.arange(nkz + 1), -np.arange(nkz, 0, -1)]) * (2 * np.pi / p.lz)
    kx = np.arange(nkx + 1) * (2 * np.pi / p.lx)
    KY, KZ, KX = np.meshgrid(ky, kz, kx, indexing="ij")
    kk = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    spec = kk ** 4 * np.exp(-2.0 * (kk / k0) ** 2)
    amp = np.sqrt(np.where(kk > 0, spec / np.maximum(kk, 1e-30) ** 2, 0.0))
    c = [amp * np.exp(2j * np.pi * rng.random(kk.shape)) * rng.standard_normal(kk.shape)
         for _ in range(3)]
    # solenoidal projection u -= k (k.u)/|k|^2
    with np.errstate(invalid="ignore", divide="ignore"):
        kd = (KX * c[0] + KY * c[1] + KZ * c[2]) / np.where(kk > 0, kk ** 2, 1.0)
    c = [c[0] - KX * kd, c[1] - KY * kd, c[2] - KZ * kd]
    # Hermitian symmetry on the kx = 0 plane: value(-ky,-kz) = conj(value(ky,kz))
    nyt, nzt = 2 * nky + 1, 2 * nkz + 1
    iy = np.array([(nyt - j) % nyt for j in range(nyt)])
    iz = np.array([(nzt - k) % nzt for k in range(nzt)])
    for a in c:
        a0 = a[:, :, 0]
        a[:, :, 0] = 0.5 * (a0 + np.conj(a0[iy][:, iz]))
        a[0, 0, 0] = 0.0
    e = sum(np.sum(np.abs(a[:, :, 0]) ** 2) + 2 * np.sum(np.abs(a[:, :, 1:]) ** 2) for a in c)
    scale = u_rms * np.sqrt(3.0 / max(e, 1e-300))
    return [a * scale for a in c]


def ensemble_kh_params(rng: np.random.Generator, base: Params):
    """One case of the served KH ensemble: NX in {64,128,256}, NZ in {16,32,64},
    NY in {33,65,129}; Re ~ U[500,5000]; Ri ~ U[0.05,0.25]."""
    nx = int(rng.choice([64, 128, 256]))
    nz = int(rng.choice([16, 32, 64]))
    ny = int(rng.choice([33, 65, 129]))
    re = float(rng.uniform(500, 5000))
    ri = float(rng.uniform(0.05, 0.25))
    q = base.replace(nx=nx, ny=ny, nz=nz, nu=1.0 / re)
    q.ri = list(q.ri)
    q.ri[0] = ri
    return q


def to_spectral_chan(phys: np.ndarray, p: Params) -> np.ndarray:
    """FFT_XZ_TO_FOURIER of physical planes [NY+2][NZ][NX] on the host with
    numpy (the packing and scaling of for/mpi.f:1530-1611): retained modes
    [NY+2][TNKZ+1][NKX+1].  For preparing initial states off the GPU."""
    t = np.fft.fft(np.fft.rfft(phys, axis=2)[:, :, : p.nkx + 1] / p.nx, axis=1) / p.nz
    out = np.zeros((phys.shape[0], 2 * p.nkz + 1, p.nkx + 1), dtype=np.complex128)
    out[:, : p.nkz + 1] = t[:, : p.nkz + 1]
    out[:, p.nkz + 1:] = t[:, p.nz - p.nkz:]
    return out


def kh_state(p: Params, gy: np.ndarray, seed: int = 1, kick: float = 1e-3) -> dict:
    """Spectral KH initial state (CU1..3, CP = 0, CTHn) for the ensemble
    server; the server's prepare step applies the BCs and REM_DIV_CHAN."""
    u1, u2, u3, th = kh_shear_layer(p, gy, seed=seed, kick=kick)
    st = {"CU1": to_spectral_chan(u1, p), "CU2": to_spectral_chan(u2, p),
          "CU3": to_spectral_chan(u3, p),
          "CP": np.zeros((p.ny + 2, 2 * p.nkz + 1, p.nkx + 1), dtype=np.complex128)}
    for n in range(p.n_th):
        st[f"CTH{n}"] = to_spectral_chan(th[n], p)
    return st
