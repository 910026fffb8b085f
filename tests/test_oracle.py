"""Pins of the CPU oracle (no GPU).

The reference ships no tests or golden vectors and cannot be built here, so
the oracle is pinned against: numpy.fft (FFTW's published sign and scaling
conventions), dense linear algebra (the Thomas routines), the divergence-free
constraint REM_DIV_CHAN / REM_DIV_PER enforce, exact discrete solutions of the
RK3/CN scheme (a decaying Fourier mode; the laminar Poiseuille profile), and
the reference's own KH grid fixture (tests/test_inputs.py).
"""
import math

import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics
from diablo_b200.grid import uniform_grid
from diablo_b200.params import Params


@pytest.mark.parametrize("n", [1, 2, 3, 7, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512])
def test_fft1d_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(O.fft1d(x, -1), np.fft.fft(x), rtol=0, atol=1e-12 * n)
    np.testing.assert_allclose(O.fft1d(x, +1), n * np.fft.ifft(x), rtol=0, atol=1e-12 * n)


def numpy_xz_to_fourier(phys, nkx, nkz):
    """Independent statement of FFT_XZ_TO_FOURIER (for/mpi.f:1530-1611)."""
    ny2, nz, nx = phys.shape
    t = np.fft.fft(np.fft.rfft(phys, axis=2)[:, :, : nkx + 1] / nx, axis=1) / nz
    out = np.zeros((ny2, 2 * nkz + 1, nkx + 1), dtype=complex)
    out[:, : nkz + 1] = t[:, : nkz + 1]
    out[:, nkz + 1:] = t[:, nz - nkz:]
    return out


def numpy_xz_to_physical(spec, nx, nz):
    ny2, nzt, nkxp = spec.shape
    nkz = (nzt - 1) // 2
    full = np.zeros((ny2, nz, nx // 2 + 1), dtype=complex)
    full[:, : nkz + 1, :nkxp] = spec[:, : nkz + 1]
    full[:, nz - nkz:, :nkxp] = spec[:, nkz + 1:]
    t = np.fft.ifft(full, axis=1) * nz
    t[:, :, 0] = t[:, :, 0].real          # c2r ignores Im of the x-DC bin
    return np.fft.irfft(t, n=nx, axis=2) * nx


@pytest.mark.parametrize("nx,nz,ny", [(16, 16, 5), (32, 48, 9), (64, 24, 6)])
def test_xz_transforms_match_numpy(nx, nz, ny):
    p = Params(nx=nx, ny=ny, nz=nz, lx=1.0, lz=1.0)
    o = O.Oracle(p, uniform_grid(ny, -1, 1))
    rng = np.random.default_rng(1)
    phys = rng.standard_normal(p.phys_shape())
    spec = o.to_fourier(phys)
    ref = numpy_xz_to_fourier(phys, p.nkx, p.nkz)
    np.testing.assert_allclose(spec, ref, atol=1e-14 * np.abs(ref).max())
    back = o.to_physical(spec)
    np.testing.assert_allclose(back, numpy_xz_to_physical(spec, nx, nz), atol=1e-12)
    # spectral -> physical -> spectral is the identity on retained modes
    np.testing.assert_allclose(o.to_fourier(back), spec, atol=1e-13 * np.abs(spec).max())


def test_xzy_transform_matches_numpy():
    n = 24
    p = Params(nx=n, ny=n, nz=n, num_per_dir=3, lx=1, ly=1, lz=1)
    o = O.Oracle(p, None)
    rng = np.random.default_rng(2)
    phys = rng.standard_normal(p.phys_shape())
    spec = o.to_fourier(phys)
    full = np.fft.fftn(np.fft.rfft(phys, axis=2), axes=(0, 1)) / n ** 3
    nk = n // 3
    idx = np.r_[0: nk + 1, n - nk: n]
    ref = full[np.ix_(idx, idx, np.arange(nk + 1))]
    np.testing.assert_allclose(spec, ref, atol=1e-14 * np.abs(ref).max())


@pytest.mark.parametrize("kind", ["real", "complex"])
def test_thomas_matches_dense(kind):
    rng = np.random.default_rng(3)
    ny, nx = 20, 6
    a = rng.uniform(-1, 1, (ny + 1, nx + 1))
    c = rng.uniform(-1, 1, (ny + 1, nx + 1))
    b = 4 + rng.uniform(0, 1, (ny + 1, nx + 1))
    if kind == "real":
        g = rng.standard_normal((ny + 1, nx + 1))
        x = O.thomas_real(a, b, c, g, ny, nx)
    else:
        g = rng.standard_normal((ny + 1, nx + 1)) + 1j * rng.standard_normal((ny + 1, nx + 1))
        x = O.thomas_complex(a, b, c, g, ny, nx)
    for i in range(nx + 1):
        m = np.diag(b[:, i]) + np.diag(a[1:, i], -1) + np.diag(c[:-1, i], 1)
        np.testing.assert_allclose(x[:, i], np.linalg.solve(m, g[:, i]), rtol=1e-12, atol=1e-12)


def test_rem_div_chan_divergence_free():
    p, gy = configs.channel_re180(nx=32, ny=33, nz=32)
    o = O.Oracle(p, gy)
    u1, u2, u3, _ = ics.channel_laminar(p, gy, seed=5)
    o.create_flow_chan(u1, u2, u3, None)
    scale = max(np.abs(o.get("CU1")).max(), 1.0) * p.nkx * 2 * math.pi / p.lx
    assert o.div_max() < 1e-13 * scale


def test_periodic_mode_decays_exactly():
    """u1 = sin(y) (a shear mode): the nonlinear term vanishes and each RK3
    substep multiplies the mode by (1 - nu h k^2/2)/(1 + nu h k^2/2)."""
    n = 24
    p = Params(nx=n, ny=n, nz=n, num_per_dir=3, nu=0.05, lx=2 * math.pi, ly=2 * math.pi,
               lz=2 * math.pi, delta_t=0.01)
    o = O.Oracle(p, None)
    y = np.arange(n) * 2 * math.pi / n
    u1 = np.sin(y)[:, None, None] * np.ones((n, n, n))
    z = np.zeros((n, n, n))
    o.create_flow_per(u1, z, z)
    a0 = o.get("CU1")[1, 0, 0]
    nsteps = 10
    for s in range(nsteps):
        o.step(s + 1)
    amp = 1.0
    for _ in range(nsteps):
        for h in (8 / 15, 2 / 15, 5 / 15):
            t = p.nu * h * p.delta_t / 2 * 1.0
            amp *= (1 - t) / (1 + t)
    a1 = o.get("CU1")[1, 0, 0]
    assert abs(a1 - a0 * amp) < 1e-14
    others = o.get("CU1").copy()
    others[1, 0, 0] = others[-1, 0, 0] = 0
    assert np.abs(others).max() < 1e-15


def test_poiseuille_is_a_fixed_point():
    """Laminar channel under constant pressure gradient: U = (1 - y^2)/(2 nu)
    is an exact steady state of the discrete CN/FD operator on a uniform grid
    (second differences of a quadratic are exact)."""
    ny = 17
    gy = uniform_grid(ny, -1.0, 1.0)
    p = Params(nx=16, ny=ny, nz=16, num_per_dir=2, nu=0.1, lx=2.0, ly=2.0, lz=2.0,
               delta_t=0.05, f_type=1, px0=-1.0, u_bc_ymin=0, u_bc_ymax=0, v_bc_ymin=0,
               v_bc_ymax=0, w_bc_ymin=0, w_bc_ymax=0)
    o = O.Oracle(p, gy)
    _, gyf, _, _ = (lambda g: (None, 0.5 * (g[:-1] + g[1:]), None, None))(gy)
    from diablo_b200.grid import grid_metrics
    _, GYF, _, _ = grid_metrics(gy)
    u1 = np.zeros(p.phys_shape())
    u1[:] = ((1 - GYF ** 2) / (2 * p.nu))[:, None, None]
    z = np.zeros(p.phys_shape())
    o.create_flow_chan(u1, z, z, None)
    before = o.get("CU1")[:, 0, 0].real.copy()
    for s in range(5):
        o.step(s + 1)
    after = o.get("CU1")[:, 0, 0].real
    np.testing.assert_allclose(after[1: ny + 1], before[1: ny + 1], rtol=0, atol=1e-11)
    assert np.abs(o.get("CU2")).max() < 1e-12


def test_kh_oracle_runs_and_conserves_structure():
    p, gy = configs.kh_shear_layer(nx=32, ny=33, nz=16)
    o = O.Oracle(p, gy)
    u1, u2, u3, th = ics.kh_shear_layer(p, gy, seed=1)
    o.create_flow_chan(u1, u2, u3, th)
    s0 = o.stats()
    for s in range(5):
        o.step(s + 1)
    s1 = o.stats()
    assert np.isfinite(s1["ke"]) and abs(s1["ke"] - s0["ke"]) < 1e-3 * s0["ke"]
    assert s1["div_max"] < 1e-12


def test_host_spectral_ic_matches_oracle_transform():
    """ics.to_spectral_chan (numpy, for preparing server requests) equals the
    oracle's FFT_XZ_TO_FOURIER."""
    p, gy = configs.kh_shear_layer(nx=32, ny=17, nz=16)
    o = O.Oracle(p, gy)
    rng = np.random.default_rng(12)
    phys = rng.standard_normal(p.phys_shape())
    np.testing.assert_allclose(ics.to_spectral_chan(phys, p), o.to_fourier(phys), rtol=0,
                               atol=1e-15)
