"""Channel LES (constant Smagorinsky) on the device against the oracle
(needs a B200).

The device keeps the fused spectral nonlinear stage and adds the subgrid
model around it; the oracle follows the reference's physical-space order
(for/les.f:1-275, for/channel.f:299-372,631-659,748-1029).  Parity bar: FP64,
relative L2 <= 1e-11 per field after the steps below, NU_T to 1e-11 of its
largest value, and the projected velocity divergence-free to 1e-12.
"""
import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics

pytestmark = pytest.mark.gpu

TOL = 1e-11


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def start(p, gy, maker, seed, **kw):
    from diablo_b200.solver import Channel
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = maker(p, gy, seed=seed, **kw)
    ref.create_flow_chan(u1, u2, u3, th if p.n_th else None)
    ch = Channel(p, gy)
    ch.set_state(ref.state())
    ch.set_time(0.0, p.delta_t)
    return ref, ch


def compare(ref, ch, p, tol=TOL):
    bad = {}
    names = ["CU1", "CU2", "CU3", "CP"] + [f"CTH{n}" for n in range(p.n_th)]
    for n in names:
        r = rel(ch.get_field(n), ref.get(n))
        if not r <= tol:
            bad[n] = r
    a, b = ch.nu_t(), ref.nu_t()
    e = np.abs(a - b).max()
    if not e <= tol * np.abs(b).max():
        bad["NU_T"] = e
    assert not bad, bad
    return np.abs(b).max()


def kh_les(**kw):
    p, gy = configs.kh_shear_layer(nx=64, ny=33, nz=32)
    p = p.replace(les=1, les_model_type=1, n_th=2, delta_t=0.02, **kw)
    p.ri = [0.1, 0.05, 0, 0]
    p.pr = [1.0, 0.7, 1, 1]
    p.th_bc_ymin = [0, 1, 0, 0]      # the second scalar has Neumann walls: JSTART_TH = 1
    p.th_bc_ymax = [0, 1, 0, 0]
    p.th_bc_ymin_c1 = [-1.0, 0.0, 0, 0]
    p.th_bc_ymax_c1 = [1.0, 0.0, 0, 0]
    return p, gy


def test_kh_les_neumann_walls_two_scalars():
    p, gy = kh_les()
    ref, ch = start(p, gy, ics.kh_shear_layer, seed=21, kick=0.3)
    for s in range(1, 9):
        ref.step(s)
        ch.step(s)
    assert compare(ref, ch, p) > 1e-4          # the model is doing work
    assert ch.stats()["div_max"] < 1e-12
    ch.close()


def test_channel_les_no_slip_with_courant():
    p, gy = configs.channel_re180(nx=64, ny=65, nz=48)
    p = p.replace(les=1, les_model_type=1)
    ref, ch = start(p, gy, ics.channel_laminar, seed=22)
    for s in range(1, 6):
        ref.step(s)
        ch.step(s)
    assert abs(ch.get_time()[1] - ref.get_time()[1]) <= 1e-13 * ref.get_time()[1]
    assert compare(ref, ch, p) > 1e-6
    assert ch.stats()["div_max"] < 1e-12
    ch.close()


def test_spin_up_then_model():
    from diablo_b200.solver import Channel
    p, gy = kh_les(create_new_flow=1)
    ref, ch = start(p, gy, ics.kh_shear_layer, seed=23, kick=0.3)
    dns = Channel(p.replace(les=0), gy)
    dns.set_state(ref.state())
    dns.set_time(0.0, p.delta_t)
    for s in (1, 2):
        ref.step(s)
        ch.step(s)
        dns.step(s)
    # during the first 100 steps of a new flow the LES handle runs the DNS
    for n in ("CU1", "CU2", "CU3", "CP", "CTH0", "CTH1"):
        assert np.array_equal(ch.get_field(n), dns.get_field(n)), n
    for s in (101, 102):
        ref.step(s)
        ch.step(s)
    compare(ref, ch, p)
    ch.close()
    dns.close()


def test_les_graph_steps_match_eager():
    from diablo_b200.solver import Channel
    p, gy = kh_les()
    ref, eager = start(p, gy, ics.kh_shear_layer, seed=24, kick=0.3)
    graph = Channel(p, gy)
    graph.set_state(ref.state())
    graph.set_time(0.0, p.delta_t)
    for s in range(1, 5):
        eager.step(s)
    graph.steps(1, 4)
    for n in ("CU1", "CU2", "CU3", "CP", "CTH0", "CTH1"):
        assert np.array_equal(graph.get_field(n), eager.get_field(n)), n
    eager.close()
    graph.close()


@pytest.mark.parametrize("shape", [(64, 33, 32), (128, 65, 16), (128, 33, 128), (96, 17, 48)])
def test_les_plane_transforms_match_staged(shape):
    """The whole-plane transform kernels (one launch per direction, the z
    columns held in shared memory) against the staged pair of launches
    through the half-physical array: same passes and twiddles, so the LES
    steps agree to round-off (bitwise where the compiler contracts the
    same multiply-adds); both against the oracle."""
    from diablo_b200.solver import Channel
    nx, ny, nz = shape
    p, gy = configs.kh_shear_layer(nx=nx, ny=ny, nz=nz)
    p = p.replace(les=1, les_model_type=1, n_th=1, delta_t=0.02)
    ref, fused = start(p, gy, ics.kh_shear_layer, seed=26, kick=0.3)
    staged = Channel(p, gy)
    staged.set_state(ref.state())
    staged.set_time(0.0, p.delta_t)
    staged.tune_set(plane_xz=0)
    assert fused.tune_get()["plane_xz"] == 1 and staged.tune_get()["plane_xz"] == 0
    for s in range(1, 4):
        ref.step(s)
        fused.step(s)
        staged.step(s)
    for n in ("CU1", "CU2", "CU3", "CP", "CTH0"):
        a, b = fused.get_field(n), staged.get_field(n)
        assert rel(a, b) <= 1e-14, (n, rel(a, b))
    same = all(np.array_equal(fused.get_field(n), staged.get_field(n))
               for n in ("CU1", "CU2", "CU3", "CP", "CTH0"))
    print(f"PLANE_XZ {shape} bitwise={same}")
    compare(ref, fused, p)
    fused.close()
    staged.close()


@pytest.mark.parametrize("bad", [dict(les_model_type=2), dict(v_bc_ymax=1)])
def test_les_refusals(bad):
    from diablo_b200.solver import Channel
    from diablo_b200._lib import DiabloError
    p, gy = configs.kh_shear_layer(nx=64, ny=33, nz=32)
    with pytest.raises(DiabloError):
        Channel(p.replace(les=1, **bad), gy)


def test_les_plane_means_match_oracle(tmp_path):
    from diablo_b200 import stats_io
    p, gy = kh_les()
    ref, ch = start(p, gy, ics.kh_shear_layer, seed=25, kick=0.3)
    for s in (1, 2, 3):
        ref.step(s)
        ch.step(s)
    ref.les_stats_request()
    ch.les_stats_request()
    ref.rk_chan_1(4, 1)
    ch.rk_chan_1(4, 1)
    got, want = ch.les_stats(), ref.les_stats()
    for k in ("nu_sgs", "eps_sgs1"):
        g, w = got[k][1:-1], want[k][1:-1]
        assert np.abs(w).max() > 0, k
        assert np.abs(g - w).max() <= 1e-11 * np.abs(w).max() + 1e-15, k
    path = tmp_path / "mean_les.txt"
    stats_io.write_mean_les(str(path), got, ch.GYF, 4, 0.06, p.delta_t)
    assert len(open(path).read().splitlines()) == 1 + 2 * p.ny
    ch.close()


@pytest.mark.parametrize("case", ["kh", "channel"])
def test_les_mixed_precision(case):
    """Mixed precision (FP32 nonlinear transforms and products) with the
    subgrid model, whose own stages and the column solves stay FP64: the
    mixed-precision bar, relative L2 <= 1e-5 against the FP64 oracle."""
    from diablo_b200.solver import Channel
    if case == "kh":
        p, gy = kh_les()
        maker, kw, nsteps = ics.kh_shear_layer, {"kick": 0.3}, 8
    else:
        p, gy = configs.channel_re180(nx=64, ny=65, nz=48)
        p = p.replace(les=1, les_model_type=1)
        maker, kw, nsteps = ics.channel_laminar, {}, 5
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = maker(p, gy, seed=26, **kw)
    ref.create_flow_chan(u1, u2, u3, th if p.n_th else None)
    g = Channel(p.replace(precision=1), gy)
    g.set_state(ref.state())
    g.set_time(0.0, p.delta_t)
    for s in range(1, nsteps + 1):
        ref.step(s)
        g.steps(s, 1)
    names = ["CU1", "CU2", "CU3"] + [f"CTH{n}" for n in range(p.n_th)]
    err = {n: rel(g.get_field(n), ref.get(n)) for n in names}
    assert all(v <= 1e-5 for v in err.values()), err
    assert g.stats()["div_max"] < 1e-12
    g.close()


def test_tkebudget_chan_les_matches_oracle():
    p, gy = kh_les()
    ref, ch = start(p, gy, ics.kh_shear_layer, seed=27, kick=0.3)
    for s in (1, 2, 3):
        ref.step(s)
        ch.step(s)
    want, got = ref.tkebudget_chan_les(), ch.les_tke()
    # row 1 is 0/0 in both (DYF(0) unset), rows 2..NY are sums over a plane
    assert np.isnan(want[1]) and np.isnan(got[1])
    w, g = want[2:p.ny + 1], got[2:p.ny + 1]
    assert np.abs(g - w).max() <= 1e-11 * np.abs(w).max() + 1e-15
    # both applied APPLY_BC_VEL to their state first
    for n in ("CU1", "CU2", "CU3"):
        assert rel(ch.get_field(n), ref.get(n)) <= TOL, n
    ch.close()


def test_kh_test_les_100_steps():
    """The reference's own KH_test run (KH_test/input*.dat, grid.h5: 128x65x16
    stretched, CFL 0.5 with COURANT every step, Neumann scalar, constant
    Smagorinsky from the first step) for 100 steps against the oracle."""
    p, gy = configs.kh_les()
    ref, ch = start(p, gy, ics.kh_shear_layer, seed=28, kick=0.1)
    for s in range(1, 101):
        ref.step(s)
        ch.steps(s, 1)
    t_ref, dt_ref = ref.get_time()
    t, dt = ch.get_time()
    assert abs(t - t_ref) <= 1e-12 * t_ref and abs(dt - dt_ref) <= 1e-12 * dt_ref
    compare(ref, ch, p)
    assert ch.stats()["div_max"] < 1e-12
    ch.close()
