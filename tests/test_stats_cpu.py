"""SAVE_STATS_CHAN statistics on the CPU (no GPU needed).

* The plane sums the device kernel forms by the discrete Parseval identity
  (csrc/chan_stats.cu), restated in numpy from the spectral state, against
  the oracle's physical-space restatement of for/save_stats.f: this checks
  the method itself, including the reference's mean shift in the dv/dy term
  and the real part of the (0,0) mode.  Tolerance: 1e-12 of each profile's
  largest magnitude plus 1e-15 absolute.  The physical-space sums subtract
  O(1) plane means from O(1) point values, so a fluctuation of 1e-6 (the KH
  seed noise) carries ~1e-16 absolute round-off there, which is 1e-11
  relative; the spectral sums never form that difference.
* The reference's text formats (diablo_b200.stats_io) round-trip.
"""
import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics, stats_io
from diablo_b200.grid import create_grid

ATOL = 1e-15


def parseval_profiles(ref, p):
    ref.apply_bc_vel()
    GY, GYF, DY, DYF = ref.grid()
    nkx, nkz = p.nx // 3, p.nz // 3
    KX = np.arange(nkx + 1) * 2 * np.pi / p.lx
    KZ = np.concatenate([np.arange(nkz + 1), -np.arange(nkz, 0, -1)]) * 2 * np.pi / p.lz
    w = np.where(np.arange(nkx + 1) == 0, 1.0, 2.0)[None, None, :]
    kx2 = (KX ** 2)[None, None, :]
    kz2 = (KZ ** 2)[None, :, None]

    def real_mean(a):
        b = a.copy()
        b[:, 0, 0] = b[:, 0, 0].real
        return b

    def fl(a):
        b = a.copy()
        b[:, 0, 0] = 0
        return b

    def S(x):  # plane sums
        return (w * x).sum(axis=(1, 2)).real

    n2 = lambda x: np.abs(x) ** 2
    dot = lambda a, b: (a * np.conj(b)).real
    a1, a2, a3 = (real_mean(ref.get(n)) for n in ("CU1", "CU2", "CU3"))
    ny, L = p.ny, p.ny + 2
    J = np.arange(1, ny + 1)
    out = {k: np.zeros(L) for k in O.PROFILES}
    out["ume"], out["vme"], out["wme"] = a1[:, 0, 0].real, a2[:, 0, 0].real, a3[:, 0, 0].real
    out["cp"] = ref.get("CP")[:, 0, 0].real
    f1, f2, f3 = fl(a1), fl(a2), fl(a3)
    A22 = S(n2(f2))
    out["urms"][J] = np.sqrt(S(n2(f1))[J])
    out["vrms"][J] = np.sqrt(0.5 * (A22[J] + A22[J + 1]))
    out["wrms"][J] = np.sqrt(S(n2(f3))[J])
    X12, X32 = S(dot(f1, f2)), S(dot(f3, f2))
    X12m = np.zeros(L); X32m = np.zeros(L)
    X12m[J] = S(dot(f1[J - 1], f2[J]))
    X32m[J] = S(dot(f3[J - 1], f2[J]))
    out["uv"][J] = (DYF[J - 1] * X12[J] + DYF[J] * X12m[J]) / (2 * DY[J])
    out["wv"][J] = (DYF[J - 1] * X32[J] + DYF[J] * X32m[J]) / (2 * DY[J])
    out["uw"][J] = S(dot(f1, f3))[J]
    out["dudy"][J] = (out["ume"][J] - out["ume"][J - 1]) / (GYF[J] - GYF[J - 1])
    out["dwdy"][J] = (out["wme"][J] - out["wme"][J - 1]) / (GYF[J] - GYF[J - 1])
    d1, d3 = a1[J + 1] - a1[J - 1], a3[J + 1] - a3[J - 1]
    out["shear"][J] = S(n2(d1) + n2(d3)) / (2 * DYF[J]) ** 2
    i2f = (1 / (2 * DYF[J]))[:, None, None]
    v2 = 0.5 * (a2[J + 1] + a2[J])
    ikz = 1j * KZ[None, :, None]
    ikx = 1j * KX[None, None, :]
    out["omega_x"][J] = np.sqrt(S(n2(d3 * i2f - ikz * v2)))
    out["omega_y"][J] = np.sqrt(S(n2(ikz * a1[J] - ikx * a3[J])))
    out["omega_z"][J] = np.sqrt(S(n2(ikx * v2 - d1 * i2f)))
    E = {nm: S(k2 * n2(a)) for nm, k2, a in (("ux", kx2, a1), ("vx", kx2, a2), ("wx", kx2, a3),
                                              ("uz", kz2, a1), ("vz", kz2, a2), ("wz", kz2, a3))}
    Euy = np.zeros(L); Ewy = np.zeros(L); Evy = np.zeros(L)
    Euy[J] = S(n2(f1[J] - f1[J - 1]))
    Ewy[J] = S(n2(f3[J] - f3[J - 1]))
    dv = a2[J + 1] - a2[J - 1]
    dv[:, 0, 0] = a2[J + 1, 0, 0].real - a2[J, 0, 0].real
    Evy[J] = S(n2(dv))
    for j in range(2, ny):
        ip = lambda q: (DYF[j - 1] * q[j] + DYF[j] * q[j - 1]) / (2 * DY[j])
        e = (ip(E["ux"]) + E["vx"][j] + Euy[j] / DY[j] ** 2 + ip(E["wx"]) + ip(E["uz"])
             + Evy[j] / (GY[j + 1] - GY[j - 1]) ** 2 + Ewy[j] / DY[j] ** 2 + E["vz"][j]
             + ip(E["wz"]))
        out["epsilon"][j] = p.nu * e
    for k in O.PROFILES_TH:
        out[k] = np.zeros((p.n_th, L))
    for n in range(p.n_th):
        t = real_mean(ref.get(f"CTH{n}"))
        out["thme"][n] = t[:, 0, 0].real
        ft = fl(t)
        out["thrms"][n][J] = np.sqrt(S(n2(ft))[J])
        out["thv"][n][J] = S(dot(ft[J], 0.5 * (f2[J] + f2[J + 1])))
        out["dthdy"][n][J] = (out["thme"][n][J] - out["thme"][n][J - 1]) / (GYF[J] - GYF[J - 1])
        g = (GYF[J + 1] - GYF[J - 1])
        out["pe_diss"][n][J] = S((kx2 + kz2) * n2(t))[J] + S(n2(t[J + 1] - t[J - 1])) / g ** 2
    return out


@pytest.mark.parametrize("case", ["kh_two_scalars", "re180_stretched_small"])
def test_parseval_sums_match_physical_space(case):
    if case == "kh_two_scalars":
        p, gy = configs.kh_shear_layer(nx=32, ny=25, nz=16)
        p = p.replace(n_th=2)
        p.ri = [0.1, -0.05, 0, 0]
        p.pr = [1.0, 0.7, 1, 1]
        maker = ics.kh_shear_layer
    else:
        p, gy = configs.channel_re180(nx=32, ny=33, nz=24)
        maker = ics.channel_laminar
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = maker(p, gy, seed=5)
    ref.create_flow_chan(u1, u2, u3, th if p.n_th else None)
    for s in range(1, 4):
        ref.step(s)
    got = parseval_profiles(ref, p)
    want = ref.save_stats_chan()
    for k in O.PROFILES:
        sl = slice(2, -2) if k == "epsilon" else slice(1, -1)
        g, w = got[k][sl], np.asarray(want[k])[sl]
        assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max() + ATOL, k
    for k in O.PROFILES_TH:
        for n in range(p.n_th):
            g, w = got[k][n][1:-1], np.asarray(want[k][n])[1:-1]
            assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max() + ATOL, (k, n)


def test_stats_text_formats(tmp_path):
    p, gy = configs.kh_shear_layer(nx=32, ny=17, nz=16)
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = ics.kh_shear_layer(p, gy, seed=2)
    ref.create_flow_chan(u1, u2, u3, th)
    ref.step(1)
    st = ref.save_stats_chan()
    L = p.ny + 2
    m = {"ubar": np.zeros(L), "vbar": np.zeros(L), "wbar": np.zeros(L),
         "thbar": np.zeros((p.n_th, L))}
    ref.stats_means_update(1, m["ubar"], m["vbar"], m["wbar"], m["thbar"])
    gyf = ref.grid()[1]
    stats_io.write_mean(str(tmp_path / "mean.txt"), st, gyf, 1, 0.01, p.delta_t)
    stats_io.write_mean_th(str(tmp_path / "mean_th.txt"), st, gyf, 1, 0.01, p.delta_t)
    stats_io.write_tke(str(tmp_path / "tke.txt"), st, gyf, 1, 0.01, p.delta_t)
    stats_io.write_stats_final(str(tmp_path / "stats.txt"), m, gyf)
    rows = np.loadtxt(tmp_path / "mean.txt", skiprows=2)
    assert rows.shape == (p.ny, 18)
    assert np.array_equal(rows[:, 0], np.arange(1, p.ny + 1))
    assert np.allclose(rows[:, 2], st["ume"][1:-1], rtol=0, atol=1e-19)
    assert np.allclose(rows[:, 3], 0.5 * (st["vme"][2:] + st["vme"][1:-1]), rtol=0, atol=1e-19)
    assert np.allclose(rows[:, 17], st["omega_z"][1:-1], rtol=0, atol=1e-19)
    th = np.loadtxt(tmp_path / "mean_th.txt", skiprows=2)
    assert th.shape == (p.ny * p.n_th, 7)
    assert np.allclose(th[:, 6], st["pe_diss"][0][1:-1], rtol=0, atol=1e-19)
    tke = np.loadtxt(tmp_path / "tke.txt", skiprows=1)
    assert tke.shape == (p.ny - 2, 3)
    assert np.allclose(tke[:, 2], st["epsilon"][2:-2], rtol=0, atol=1e-9)
    lines = (tmp_path / "stats.txt").read_text().splitlines()
    assert len(lines) == p.ny * (1 + p.n_th)
    assert len(lines[0].split(",")) == 5 and len(lines[-1].split(",")) == 3
    # first sample: the running mean is the sample (weights 1 and 0)
    assert np.array_equal(m["ubar"][1:-1], st["ume"][1:-1])
