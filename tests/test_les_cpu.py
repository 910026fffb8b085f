"""The oracle's LES (constant Smagorinsky, for/les.f:1-275) on CPU.

Pins: NU_T of one substep against an independent numpy statement of
compute_strain_chan, |S| at GY points, the filter width and GHOST_LES_MPI;
the spin-up rule (no subgrid model during the first 100 steps of a new flow,
for/channel.f:303); a parallel shear flow, whose strain the model removes
with the mean shear, steps exactly like the DNS; and the projection still
leaves a divergence-free field.
"""
import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics


def les_case(nx=32, ny=25, nz=16, kick=0.3, seed=11, **kw):
    p, gy = configs.kh_shear_layer(nx=nx, ny=ny, nz=nz)
    p = p.replace(les=1, les_model_type=1, variable_dt=0, delta_t=0.02, **kw)
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = ics.kh_shear_layer(p, gy, seed=seed, kick=kick)
    ref.create_flow_chan(u1, u2, u3, th)
    return p, gy, ref


def to_phys(spec, nx, nz):
    """FFT_XZ_TO_PHYSICAL (for/mpi.f:1613-1674) by numpy: retained modes only."""
    ny2, nzt, nkxp = spec.shape
    nkz = (nzt - 1) // 2
    t = np.zeros((ny2, nz, nx // 2 + 1), dtype=complex)
    t[:, : nkz + 1, :nkxp] = spec[:, : nkz + 1]
    t[:, nz - nkz:, :nkxp] = spec[:, nkz + 1:]
    t = np.fft.ifft(t, axis=1) * nz
    return np.fft.irfft(t, n=nx, axis=2) * nx


def numpy_nu_t(p, ref):
    """NU_T of les_chan from the state at the start of a substep."""
    _gy, _gyf, DY, DYF = ref.grid()
    ny = p.ny
    cu1, cu2, cu3 = (ref.get(n).copy() for n in ("CU1", "CU2", "CU3"))
    # APPLY_BC_VEL_MPI then APPLY_BC_LES (Neumann U1, U3 at both walls here)
    ref.apply_bc_vel()
    cu1, cu2, cu3 = (ref.get(n).copy() for n in ("CU1", "CU2", "CU3"))
    for c in (cu1, cu3):
        c[ny], c[ny + 1] = c[ny - 1], c[ny - 1]
        c[1], c[0] = c[2], c[2]
    nkx, nkz = p.nkx, p.nkz
    kx = 2 * np.pi / p.lx * np.arange(nkx + 1)
    kz = 2 * np.pi / p.lz * np.concatenate([np.arange(nkz + 1), -np.arange(nkz, 0, -1)])
    ikx, ikz = 1j * kx[None, None, :], 1j * kz[None, :, None]
    S = [np.zeros_like(cu1) for _ in range(6)]
    d = lambda a, j, w: (a[j] - a[j - 1]) / w[j]
    for j in range(1, ny + 1):
        S[0][j] = ikx[0] * cu1[j]
        S[1][j] = (cu2[j + 1] - cu2[j]) / DYF[j]
        S[2][j] = ikz[0] * cu3[j]
        S[4][j] = 0.5 * (ikz[0] * cu1[j] + ikx[0] * cu3[j])
    for j in range(1, ny + 2):
        S[3][j] = 0.5 * (d(cu1, j, DY) + ikx[0] * cu2[j])
        S[5][j] = 0.5 * (ikz[0] * cu2[j] + d(cu3, j, DY))
    s = [to_phys(a, p.nx, p.nz) for a in S]
    u1b, u3b = cu1[:, 0, 0].real, cu3[:, 0, 0].real
    nut = np.zeros(p.phys_shape())
    dx, dz = p.lx / p.nx, p.lz / p.nz
    for j in range(3, ny):
        w = 2 * DY[j]
        b = [(s[0][j] * DYF[j - 1] + s[0][j - 1] * DYF[j]) / w,
             s[3][j] - 0.5 * (u1b[j] - u1b[j - 1]) / DY[j],
             (s[4][j] * DYF[j - 1] + s[4][j - 1] * DYF[j]) / w,
             (s[1][j] * DYF[j - 1] + s[1][j - 1] * DYF[j]) / w,
             s[5][j] - 0.5 * (u3b[j] - u3b[j - 1]) / DY[j],
             (s[2][j] * DYF[j - 1] + s[2][j - 1] * DYF[j]) / w]
        mag = np.sqrt(2 * b[0] ** 2 + 4 * b[1] ** 2 + 4 * b[2] ** 2 + 2 * b[3] ** 2
                      + 4 * b[4] ** 2 + 2 * b[5] ** 2)
        delta2 = 0.13 ** 2 * (dx * DY[j] * 2 * dz) ** (2.0 / 3.0)
        nut[j] = delta2 * mag
    return nut


def test_nu_t_matches_numpy_statement():
    p, gy, ref = les_case()
    ref.step(1)                      # a few substeps of history
    want_ref = O.Oracle(p, gy)
    want_ref.set_state(ref.state())
    want_ref.set_time(*ref.get_time())
    want = numpy_nu_t(p, want_ref)
    ref.rk_chan_1(2, 1)
    got = ref.nu_t()
    assert np.all(got >= 0)
    for j in (0, 1, 2, p.ny, p.ny + 1):
        assert not np.any(got[j]), j
    assert np.abs(want).max() > 1e-4
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_spin_up_runs_the_dns_path():
    p, gy, les = les_case(create_new_flow=1)
    dns = O.Oracle(p.replace(les=0), gy)
    dns.set_state(les.state())
    dns.set_time(*les.get_time())
    for s in (1, 2):
        les.step(s)
        dns.step(s)
    for n in ("CU1", "CU2", "CU3", "CP", "CTH0"):
        assert np.array_equal(les.get(n), dns.get(n)), n
    # past step 100 the model runs and the flows part
    les.step(101)
    dns.step(101)
    a, b = les.get("CU1"), dns.get("CU1")
    assert np.linalg.norm(a - b) > 1e-8 * np.linalg.norm(b)
    assert les.div_max() < 1e-12


def test_parallel_shear_flow_steps_like_dns():
    # U1 = tanh(y), TH = tanh(y), no fluctuations: S_ij minus the mean shear
    # is zero, so |S| = NU_T = 0 and every subgrid term vanishes
    p, gy, les = les_case(kick=0.0)
    dns = O.Oracle(p.replace(les=0), gy)
    dns.set_state(les.state())
    dns.set_time(*les.get_time())
    for s in (1, 2):
        les.step(s)
        dns.step(s)
    assert not np.any(les.nu_t())
    # les_chan re-applies APPLY_BC_VEL every substep, so the lower ghost plane
    # of U1 follows U1(1); the DNS leaves plane 0 as the solve found it
    for n in ("CU1", "CU2", "CU3", "CTH0"):
        a, b = les.get(n)[1:], dns.get(n)[1:]
        assert np.linalg.norm(a - b) <= 1e-14 * max(np.linalg.norm(b), 1.0), n


def test_les_model_types_2_and_3_refused():
    p, gy = configs.kh_shear_layer(nx=16, ny=9, nz=8)
    with pytest.raises(ValueError, match="not supported yet in MPI"):
        O.Oracle(p.replace(les=1, les_model_type=2), gy)


def test_les_plane_means_and_mean_les_format(tmp_path):
    from diablo_b200 import stats_io
    p, gy, ref = les_case()
    ref.step(1)
    ref.les_stats_request()
    ref.rk_chan_1(2, 1)
    st = ref.les_stats()
    np.testing.assert_allclose(st["nu_sgs"], ref.nu_t().mean(axis=(1, 2)), rtol=1e-13, atol=0)
    assert np.abs(st["eps_sgs1"]).max() > 0
    with pytest.raises(ValueError):
        les_case()[2].les_stats()          # nothing recorded without a request
    _gy, gyf, _dy, _dyf = ref.grid()
    path = tmp_path / "mean_les.txt"
    stats_io.write_mean_les(str(path), st, gyf, 2, 0.04, p.delta_t)
    lines = open(path).read().splitlines()
    # header, then per row "j GYF NU_T" and, by format reversion, "EPS" alone
    assert len(lines) == 1 + 2 * p.ny
    j, y, nu = lines[1].split()
    assert int(j) == 1 and float(y) == pytest.approx(gyf[1]) and float(nu) == pytest.approx(st["nu_sgs"][1])
    assert len(lines[2]) == 31 and float(lines[2]) == pytest.approx(st["eps_sgs1"][1], abs=1e-20)


def test_tkebudget_chan_les_and_tke_les_format(tmp_path):
    import warnings
    from diablo_b200 import stats_io
    p, gy, ref = les_case()
    ref.step(1)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        eps = ref.tkebudget_chan_les()
    # DYF(0) is never set in the reference: plane 1's U2 term is 0/0
    assert np.isnan(eps[1])
    assert np.all(np.isfinite(eps[2:p.ny + 1])) and np.abs(eps[2:p.ny + 1]).max() > 0
    # the model dissipates: the eddy-viscosity term removes energy overall
    assert eps[2:p.ny + 1].sum() < 0
    _gy, gyf, _dy, _dyf = ref.grid()
    path = tmp_path / "tke_les.txt"
    stats_io.write_tke_les(str(path), eps, gyf, 1, 0.02, p.delta_t)
    lines = open(path).read().splitlines()
    assert len(lines) == 1 + p.ny
    assert lines[1].split()[2] == "NaN"
    j, y, e = lines[2].split()
    assert int(j) == 2 and float(e) == pytest.approx(eps[2], rel=1e-12)
