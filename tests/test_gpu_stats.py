"""SAVE_STATS_CHAN + tkebudget_chan on the device against the oracle's
physical-space restatement (needs a B200).

The device forms every plane mean from the spectral state by the discrete
Parseval identity; the oracle transforms each field and derivative to
physical space and sums over the points as the reference does.  Profiles
agree to 1e-11 of each profile's largest magnitude plus 1e-15 absolute (the
physical-space sums subtract O(1) means from O(1) values, which leaves
~1e-16 absolute round-off on small fluctuation statistics).
"""
import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics
from diablo_b200.grid import create_grid

pytestmark = pytest.mark.gpu

TOL = 1e-11
ATOL = 1e-15


def start_pair(p, gy, maker, seed, nsteps):
    from diablo_b200.solver import Channel
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = maker(p, gy, seed=seed)
    ref.create_flow_chan(u1, u2, u3, th if p.n_th else None)
    ch = Channel(p, gy)
    ch.set_state(ref.state())
    ch.set_time(0.0, p.delta_t)
    for s in range(1, nsteps + 1):
        ref.step(s)
        ch.step(s)
    return ref, ch


def check_profiles(got, want, nth):
    bad = {}
    for k in O.PROFILES:
        g, w = np.asarray(got[k]), np.asarray(want[k])
        sl = slice(2, -2) if k == "epsilon" else slice(1, -1)
        err = np.abs(g[sl] - w[sl]).max()
        if not err <= TOL * np.abs(w[sl]).max() + ATOL:
            bad[k] = err
    for k in O.PROFILES_TH:
        for n in range(nth):
            g, w = np.asarray(got[k][n])[1:-1], np.asarray(want[k][n])[1:-1]
            err = np.abs(g - w).max()
            if not err <= TOL * np.abs(w).max() + ATOL:
                bad[f"{k}{n}"] = err
    for k in ("ubulk", "uc", "urms_b", "vrms_b", "wrms_b"):
        w = float(want[k])
        if not abs(float(got[k]) - w) <= TOL * abs(w) + ATOL:
            bad[k] = (got[k], w)
    assert not bad, bad


@pytest.mark.parametrize("case", ["re180_stretched", "kh_two_scalars", "odd_ny"])
def test_save_stats_chan_matches_oracle(case):
    if case == "re180_stretched":
        p, gy = configs.channel_re180(nx=64, ny=65, nz=48)
        maker, nsteps = ics.channel_laminar, 3
    elif case == "kh_two_scalars":
        p, gy = configs.kh_shear_layer(nx=64, ny=33, nz=32)
        p = p.replace(n_th=2)
        p.ri = [0.1, -0.05, 0, 0]
        p.pr = [1.0, 0.7, 1, 1]
        p.th_bc_ymin = [0, 1, 0, 0]
        p.th_bc_ymax = [0, 1, 0, 0]
        maker, nsteps = ics.kh_shear_layer, 5
    else:
        p, _ = configs.kh_shear_layer(nx=48, ny=41, nz=24)
        gy = create_grid(2, 41, 20.0, 1.5)
        maker, nsteps = ics.kh_shear_layer, 4
    ref, ch = start_pair(p, gy, maker, seed=6, nsteps=nsteps)
    want = ref.save_stats_chan()
    got = ch.save_stats()
    check_profiles(got, want, p.n_th)
    # both ran APPLY_BC_VEL on their state
    for nm in ["CU1", "CU2", "CU3"]:
        a, b = ch.get_field(nm), ref.get(nm)
        assert np.linalg.norm(a - b) <= 1e-11 * np.linalg.norm(b), nm
    # a second sample: the running means with REAL*4 weights
    ref.step(nsteps + 1)
    ch.step(nsteps + 1)
    want2 = ref.save_stats_chan()
    got2 = ch.save_stats()
    check_profiles(got2, want2, p.n_th)
    L = p.ny + 2
    ub, vb, wb = np.zeros(L), np.zeros(L), np.zeros(L)
    thb = np.zeros((max(p.n_th, 1), L))
    for k, st in enumerate((want, want2), start=1):
        for j in range(1, p.ny + 1):
            w1 = float(np.float32(1.0) / np.float32(k))
            w2 = float((np.float32(k) - np.float32(1.0)) / np.float32(k))
            ub[j] = w1 * st["ume"][j] + w2 * ub[j]
            vb[j] = w1 * st["vme"][j] + w2 * vb[j]
            wb[j] = w1 * st["wme"][j] + w2 * wb[j]
            for n in range(p.n_th):
                thb[n, j] = w1 * st["thme"][n][j] + w2 * thb[n, j]
    m = ch.stats_means()
    assert m["nsamples"] == 2
    for a, b in ((m["ubar"], ub), (m["vbar"], vb), (m["wbar"], wb)):
        assert np.abs(a - b).max() <= TOL * np.abs(b).max() + ATOL
    for n in range(p.n_th):
        assert np.abs(m["thbar"][n] - thb[n]).max() <= TOL * np.abs(thb[n]).max() + ATOL
    ch.close()
