"""Parity of the sm_100a channel path with the CPU oracle (needs a B200).

Everything is driven through the C-ABI (diablo_b200.solver wraps it with
ctypes).  Tolerances: relative L2 <= 1e-11 on U1, U2, U3 and TH (the FP64
bar), max |div u| <= 1e-12, matching KE and scalar-variance series.
"""
import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics
from diablo_b200.params import Params
from diablo_b200.grid import create_grid, uniform_grid

pytestmark = pytest.mark.gpu

TOL = 1e-11


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def channel(p, gy):
    from diablo_b200.solver import Channel
    return Channel(p, gy)


def start_pair(p, gy, maker, seed):
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = maker(p, gy, seed=seed)
    ref.create_flow_chan(u1, u2, u3, th if p.n_th else None)
    ch = channel(p, gy)
    ch.set_state(ref.state())
    ch.set_time(0.0, p.delta_t)
    return ref, ch, (u1, u2, u3, th)


def compare(ref, ch, names, tol=TOL):
    out = {}
    for k in names:
        out[k] = rel(ch.get_field(k), ref.get(k))
    bad = {k: v for k, v in out.items() if not v <= tol}
    assert not bad, out
    return out


def fields(p):
    return ["CU1", "CU2", "CU3"] + [f"CTH{n}" for n in range(p.n_th)]


# ------------------------------------------------------------------ transforms
@pytest.mark.parametrize("nx,nz,ny", [(32, 16, 9), (128, 32, 17), (48, 96, 7), (512, 384, 5),
                                      (36, 18, 6), (30, 20, 5), (80, 40, 7), (160, 120, 4)])
def test_fft_xz_matches_oracle(nx, nz, ny):
    p = Params(nx=nx, ny=ny, nz=nz, lx=1.0, lz=1.0)
    gy = uniform_grid(ny, -1, 1)
    ref = O.Oracle(p, gy)
    ch = channel(p, gy)
    rng = np.random.default_rng(nx + nz)
    phys = rng.standard_normal(p.phys_shape())
    spec_o = ref.to_fourier(phys)
    assert rel(ch.to_fourier(phys), spec_o) < 1e-14
    assert rel(ch.to_physical(spec_o), ref.to_physical(spec_o)) < 1e-14
    # partial plane ranges and reference-layout arrays
    V = np.zeros((ny + 2, nz + 2, nx + 2))
    V[:, :nz, :nx] = phys
    VV = ch.fft_xz_to_fourier(V, jmin=1, jmax=ny)
    assert rel(VV[1: ny + 1, : p.tnkz + 1, : p.nkx + 1], spec_o[1: ny + 1]) < 1e-14
    assert np.all(VV[0] == 0) and np.all(VV[:, :, p.nkx + 1:] == 0)
    ch.close()


def test_fft_xz_aliased_inplace():
    """The reference calls FFT_XZ_TO_PHYSICAL(CU1, U1, ...) on EQUIVALENCEd
    storage: one host buffer is both input and output."""
    p = Params(nx=64, ny=9, nz=32, lx=1.0, lz=1.0)
    gy = uniform_grid(9, -1, 1)
    ch = channel(p, gy)
    ref = O.Oracle(p, gy)
    rng = np.random.default_rng(4)
    phys = rng.standard_normal(p.phys_shape())
    spec = ref.to_fourier(phys)
    buf = np.zeros((p.ny + 2, p.nz + 2, p.nx // 2 + 1), dtype=np.complex128)
    buf[:, : p.tnkz + 1, : p.nkx + 1] = spec
    as_real = buf.view(np.float64).reshape(p.ny + 2, p.nz + 2, p.nx + 2)
    ch.fft_xz_to_physical(buf, as_real)          # same memory in and out
    assert rel(as_real[:, : p.nz, : p.nx], ref.to_physical(spec)) < 1e-14
    ch.close()


@pytest.mark.parametrize("kind", ["real", "complex"])
def test_thomas_matches_oracle(kind):
    from diablo_b200 import solver
    rng = np.random.default_rng(5)
    ny, nx = 64, 200
    a = rng.uniform(-1, 1, (ny + 1, nx + 1))
    c = rng.uniform(-1, 1, (ny + 1, nx + 1))
    b = 4 + rng.uniform(0, 1, (ny + 1, nx + 1))
    if kind == "real":
        g = rng.standard_normal((ny + 1, nx + 1))
        _, _, x = solver.thomas_real(a, b, c, g, ny, nx)
        xo = O.thomas_real(a, b, c, g, ny, nx)
    else:
        g = rng.standard_normal((ny + 1, nx + 1)) + 1j * rng.standard_normal((ny + 1, nx + 1))
        _, _, x = solver.thomas_complex(a, b, c, g, ny, nx)
        xo = O.thomas_complex(a, b, c, g, ny, nx)
    assert rel(x, xo) < 1e-15


# ---------------------------------------------------- IC, BCs and projection
@pytest.mark.parametrize("bc", [(0, 0, 0), (1, 0, 1), (1, 1, 1), (0, 2, 1)])
def test_bc_and_rem_div_match_oracle(bc):
    ub, vb, wb = bc
    p, gy = configs.kh_shear_layer(nx=32, ny=17, nz=16)
    p = p.replace(u_bc_ymin=ub, u_bc_ymax=ub, v_bc_ymin=vb, v_bc_ymax=vb, w_bc_ymin=wb,
                  w_bc_ymax=wb, u_bc_ymin_c1=0.3, u_bc_ymax_c1=-0.2, v_bc_ymin_c1=0.0,
                  w_bc_ymin_c1=0.1, w_bc_ymax_c1=0.05)
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = ics.kh_shear_layer(p, gy, seed=3, kick=0.05)
    ref.create_flow_chan(u1, u2, u3, th)
    ch = channel(p, gy)
    ch.create_flow(u1, u2, u3, th)
    out = compare(ref, ch, ["CU1", "CU2", "CU3", "CTH0", "CR1"], tol=1e-13)
    dg, do = ch.stats()["div_max"], ref.div_max()
    if vb == 0:
        assert dg < 1e-12
    else:
        # with V Neumann the trailing APPLY_BC_VEL rewrites CU2(NY) after the
        # projection (for/channel.f:2471-2478), so row NY-1 keeps a divergence
        # in the reference too
        assert abs(dg - do) <= 1e-9 * do + 1e-15
    ch.close()


# --------------------------------------------------------------- full steps
def test_kh_shear_layer_100_steps():
    """The CPU-runnable configuration: 128 x 65 x 32, one scalar, dt = 0.01,
    100 RK3 steps from identical seeded state; KE and scalar-variance series
    compared every 10 steps."""
    p, gy = configs.kh_shear_layer()
    ref, ch, _ = start_pair(p, gy, ics.kh_shear_layer, seed=1)
    for s in range(1, 101):
        ref.step(s)
        ch.step(s)
        if s % 10 == 0:
            so, sg = ref.stats(), ch.stats()
            assert abs(sg["ke"] - so["ke"]) <= 1e-12 * abs(so["ke"])
            assert abs(sg["th_var"][0] - so["th_var"][0]) <= 1e-9 * abs(so["th_var"][0]) + 1e-30
            assert sg["div_max"] <= 1e-12
    compare(ref, ch, fields(p))
    t_o, dt_o = ref.get_time()
    t_g, dt_g = ch.get_time()
    assert abs(t_g - t_o) < 1e-12 and dt_g == dt_o
    ch.close()


def test_channel_re180_100_steps_variable_dt():
    """128 x 129 x 128, no-slip, constant pressure gradient, COURANT every
    step (CFL 0.5): 100 RK3 steps against the oracle."""
    p, gy = configs.channel_re180()
    ref, ch, _ = start_pair(p, gy, ics.channel_laminar, seed=2)
    for s in range(1, 101):
        ref.step(s)
        ch.step(s)
    compare(ref, ch, fields(p))
    t_o, dt_o = ref.get_time()
    t_g, dt_g = ch.get_time()
    assert abs(dt_g - dt_o) <= 1e-12 * dt_o and abs(t_g - t_o) <= 1e-11 * t_o
    so, sg = ref.stats(), ch.stats()
    assert abs(sg["ke"] - so["ke"]) <= 1e-12 * so["ke"]
    assert sg["div_max"] <= 1e-12
    ch.close()


@pytest.mark.parametrize("variant", ["ftype2_rotation_gravity", "th_neumann_drho",
                                     "stretched_two_scalars", "odd_sizes", "three_scalars"])
def test_channel_variants_short(variant):
    """Paths the two configurations above do not exercise."""
    if variant == "ftype2_rotation_gravity":
        p, gy = configs.kh_shear_layer(nx=32, ny=33, nz=16)
        p = p.replace(f_type=2, px0=-0.5, omega0=3.0, amp_omega0=0.7, i_ro=0.3, grav_x=0.2,
                      grav_z=-0.1, nu_v_scale=1.3)
    elif variant == "th_neumann_drho":
        p, gy = configs.kh_shear_layer(nx=32, ny=33, nz=16)
        p = p.replace()
        p.th_bc_ymin = [1, 0, 0, 0]
        p.th_bc_ymax = [1, 0, 0, 0]
        p.th_bc_ymin_c1 = [0.2, 0, 0, 0]
        p.th_bc_ymax_c1 = [-0.1, 0, 0, 0]
        p.drhodx = [0.3, 0, 0, 0]
        p.drhodz = [-0.2, 0, 0, 0]
        p.pr = [0.7, 1, 1, 1]
    elif variant == "stretched_two_scalars":
        p, _ = configs.kh_shear_layer(nx=48, ny=41, nz=24)
        gy = create_grid(2, 41, 20.0, 1.5)
        p = p.replace(n_th=2)
        p.ri = [0.1, 0.05, 0, 0]
        p.pr = [1.0, 2.0, 1, 1]
        p.th_bc_ymin = [0, 1, 0, 0]
        p.th_bc_ymax = [0, 1, 0, 0]
        p.th_bc_ymin_c1 = [-1.0, 0.0, 0, 0]
        p.th_bc_ymax_c1 = [1.0, 0.0, 0, 0]
    elif variant == "three_scalars":                         # N_TH = 3: generic x-row path
        p, gy = configs.kh_shear_layer(nx=32, ny=25, nz=16)
        p = p.replace(n_th=3)
        p.ri = [0.1, 0.05, -0.02, 0]
        p.pr = [1.0, 2.0, 0.5, 1]
        p.th_bc_ymin = [0, 1, 0, 0]
        p.th_bc_ymax = [0, 1, 1, 0]
        p.th_bc_ymax_c1 = [0, 0, 0.2, 0]
    else:
        p, gy = configs.kh_shear_layer(nx=36, ny=11, nz=18)  # lengths without a specialisation
    ref, ch, _ = start_pair(p, gy, ics.kh_shear_layer, seed=11)
    for s in range(1, 6):
        ref.step(s)
        ch.step(s)
    compare(ref, ch, fields(p))
    compare(ref, ch, ["CF1", "CF2", "CF3"], tol=1e-10)
    # CP accumulates phi / h, and phi solves for the divergence left by the CN
    # step -- a small difference of O(1) terms -- so CP carries ~1e-10..1e-9
    # relative round-off where the velocities carry ~1e-13
    assert rel(ch.get_field("CP"), ref.get("CP")) <= 1e-8
    ch.close()


@pytest.mark.parametrize("case", ["kh_buoyant", "re180_stretched"])
def test_poisson_p_chan_matches_oracle(case):
    """POISSON_P_CHAN on a developed state: CP rows 1..NY."""
    if case == "kh_buoyant":
        p, gy = configs.kh_shear_layer(nx=64, ny=33, nz=32)
        p = p.replace(n_th=2)
        p.ri = [0.1, -0.05, 0, 0]
        p.th_bc_ymin = [0, 1, 0, 0]
        p.th_bc_ymax = [0, 1, 0, 0]
        maker = ics.kh_shear_layer
    else:
        p, gy = configs.channel_re180(nx=64, ny=65, nz=48)
        maker = ics.channel_laminar
    ref, ch, _ = start_pair(p, gy, maker, seed=4)
    for s in range(1, 4):
        ref.step(s)
        ch.step(s)
    ref.poisson_p_chan()
    ch.poisson_p_chan()
    cp_o = ref.get("CP")[1: p.ny + 1]
    cp_g = ch.get_field("CP")[1: p.ny + 1]
    assert rel(cp_g, cp_o) <= 1e-11
    compare(ref, ch, fields(p))
    ch.close()


@pytest.mark.parametrize("nx,nz", [(80, 40), (60, 30)])
def test_channel_radix5_lengths_match_oracle(nx, nz):
    """x and z lengths with a factor of 5 (FFTW takes any length; the runtime
    plans add a radix-5 pass): a stratified KH layer and a no-slip channel
    with COURANT, against the oracle."""
    p, gy = configs.kh_shear_layer(nx=nx, ny=33, nz=nz)
    ref, ch, _ = start_pair(p, gy, ics.kh_shear_layer, seed=21)
    for s in range(1, 6):
        ref.step(s)
        ch.step(s)
    compare(ref, ch, fields(p))
    ch.close()
    p, gy = configs.channel_re180(nx=nx, ny=33, nz=nz)
    ref, ch, _ = start_pair(p, gy, ics.channel_laminar, seed=22)
    for s in range(1, 6):
        ref.step(s)
        ch.step(s)
    compare(ref, ch, fields(p))
    assert abs(ch.get_time()[1] - ref.get_time()[1]) <= 1e-12 * ref.get_time()[1]
    ch.close()


@pytest.mark.parametrize("case", ["tall_ny257", "wide_512x384"])
def test_channel_large_dims_short(case):
    """NY = 257 (the CN row templates of four fields exceed 48 KB) and the
    512 x 384 plane of the Re_tau=550 configuration (x and z lengths without a
    warp-level kernel), a few steps each."""
    if case == "tall_ny257":
        p, gy = configs.kh_shear_layer(nx=32, ny=257, nz=16)
        nsteps = 4
    else:
        p, gy = configs.channel_re550(ny=17)
        nsteps = 2
    maker = ics.kh_shear_layer if case == "tall_ny257" else ics.channel_laminar
    ref, ch, _ = start_pair(p, gy, maker, seed=13)
    for s in range(1, nsteps + 1):
        ref.step(s)
        ch.step(s)
    compare(ref, ch, fields(p))
    ch.close()


def test_courant_matches_oracle():
    p, gy = configs.channel_re180(nx=64, ny=65, nz=64)
    ref, ch, _ = start_pair(p, gy, ics.channel_laminar, seed=9)
    for s in range(1, 4):
        ref.step(s)
        ch.step(s)
        assert abs(ch.get_time()[1] - ref.get_time()[1]) <= 1e-13 * ref.get_time()[1]
    ch.close()


def test_errors_are_reported_not_fatal():
    from diablo_b200.solver import DiabloError
    p, gy = configs.kh_shear_layer(nx=32, ny=17, nz=16)
    with pytest.raises(DiabloError):
        channel(p.replace(nx=28), gy)  # a factor of 7: no radix for it
    ch = channel(p, gy)
    with pytest.raises(DiabloError):
        ch.rk_chan_1(1, 4)
    bad = np.zeros(p.spec_shape(), dtype=np.complex128)
    bad[3, 2, 1] = np.nan
    ch.set_field("CU1", bad)
    with pytest.raises(DiabloError) as e:
        ch.stats()
    assert e.value.code == 5  # DG_ERR_NAN
    ch.close()


@pytest.mark.parametrize("case", ["re180_variable_dt", "kh_fixed_dt"])
def test_graph_steps_match_substep_calls(case):
    """diablo_step (graph replay after the first step) gives the same state,
    bit for bit, as three RK_CHAN_1 calls + TIME update per step."""
    if case == "re180_variable_dt":
        p, gy = configs.channel_re180(nx=64, ny=65, nz=48)
        maker = ics.channel_laminar
    else:
        p, gy = configs.kh_shear_layer(nx=64, ny=33, nz=32)
        maker = ics.kh_shear_layer
    ref, a, _ = start_pair(p, gy, maker, seed=6)
    b = channel(p, gy)
    b.set_state(ref.state())
    b.set_time(0.0, p.delta_t)
    for s in range(1, 13):
        a.step(s)
    b.steps(1, 5)
    b.steps(6, 7)
    for nm in fields(p) + ["CP"]:
        assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
    assert a.get_time() == b.get_time()
    a.close()
    b.close()


def test_autotune_restores_state_and_keeps_results():
    """dg_autotune leaves the state, TIME and DELTA_T as it found them, and
    the launch shapes it picks do not change results (bit for bit; the
    transform plan variant and the column-stage form, which change them at
    round-off level, are set the same on both sides)."""
    p, gy = configs.channel_re180(nx=64, ny=65, nz=48)
    ref, a, _ = start_pair(p, gy, ics.channel_laminar, seed=8)
    b = channel(p, gy)
    b.set_state(ref.state())
    b.set_time(0.0, p.delta_t)
    before = {nm: b.get_field(nm) for nm in fields(p) + ["CP"]}
    t0 = b.get_time()
    chosen = b.autotune(2)
    assert chosen["col_mt"] in (4, 8, 16)
    for nm, v in before.items():
        assert np.array_equal(b.get_field(nm), v), nm
    assert b.get_time() == t0
    a.tune_set(fft_plan=chosen["fft_plan"])
    for s in range(1, 6):
        a.step(s)
    b.steps(1, 5)
    for nm in fields(p) + ["CP"]:
        assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
    for mt in (4, 16):
        b.tune_set(col_mt=mt, cn_mt=20 - mt, xrow_chunk=3, ychunk=20)
        c = channel(p, gy)
        c.tune_set(fft_plan=chosen["fft_plan"])
        c.set_state(ref.state())
        c.set_time(0.0, p.delta_t)
        b.set_state(ref.state())
        b.set_time(0.0, p.delta_t)
        b.steps(1, 3)
        c.steps(1, 3)
        for nm in fields(p) + ["CP"]:
            assert np.array_equal(b.get_field(nm), c.get_field(nm)), (mt, nm)
        c.close()
    a.close()
    b.close()


@pytest.mark.parametrize("periodic", [False, True])
def test_reference_layout_round_trip(periodic):
    """diablo_set_field / diablo_get_field in the reference layout
    (0:NX/2, 0:NZ+1, planes): set reads only the retained block, get writes
    the retained block and zeros elsewhere."""
    import math
    from diablo_b200.solver import Channel, Periodic
    if periodic:
        p = Params(nx=48, ny=24, nz=36, num_per_dir=3, nu=0.01, lx=2 * math.pi,
                   ly=2 * math.pi, lz=2 * math.pi, delta_t=0.005, variable_dt=0)
        s = Periodic(p)
    else:
        p, gy = configs.kh_shear_layer(nx=48, ny=17, nz=36)
        s = Channel(p, gy)
    cmp_shape = s.get_field("CU1").shape                 # (planes, TNKZ+1, NKX+1)
    planes, nkzt, nkxp = cmp_shape
    rng = np.random.default_rng(21)
    ref = rng.standard_normal((planes, p.nz + 2, p.nx // 2 + 1)) \
        + 1j * rng.standard_normal((planes, p.nz + 2, p.nx // 2 + 1))
    s.set_field("CU2", ref, layout="reference")
    assert np.array_equal(s.get_field("CU2"), ref[:, :nkzt, :nkxp])
    back = s.get_field("CU2", layout="reference")
    want = np.zeros_like(ref)
    want[:, :nkzt, :nkxp] = ref[:, :nkzt, :nkxp]
    assert np.array_equal(back, want)
    # retained-only read: the block is written, every other entry keeps its value
    assert np.array_equal(s.get_field("CU2", layout="reference_retained"), want)
    keep = np.full(ref.shape, 7.0 - 3.0j)
    s.get_field("CU2", layout="reference_retained", out=keep)
    assert np.array_equal(keep[:, :nkzt, :nkxp], ref[:, :nkzt, :nkxp])
    keep[:, :nkzt, :nkxp] = 7.0 - 3.0j
    assert np.all(keep == 7.0 - 3.0j)
    s.set_field("CU3", ref, layout="reference_retained")
    assert np.array_equal(s.get_field("CU3"), ref[:, :nkzt, :nkxp])
    # several fields in one call, both ways
    ref2 = ref[::-1].copy()
    s.set_fields({"CU1": ref2, "CU2": ref, "CP": -ref}, layout="reference_retained")
    out = {n: np.full(ref.shape, 5.0 + 0j) for n in ("CP", "CU1", "CU2")}
    s.get_fields(out, layout="reference_retained")
    for n, a in (("CU1", ref2), ("CU2", ref), ("CP", -ref)):
        assert np.array_equal(out[n][:, :nkzt, :nkxp], a[:, :nkzt, :nkxp]), n
        assert np.all(out[n][:, nkzt:, :] == 5.0) and np.all(out[n][:, :, nkxp:] == 5.0), n
    s.close()


def test_fft_plan_variant_parity_and_tuning_cache(tmp_path):
    """The reversed-radix transform plan (DG_TUNE_FFT_PLAN = 1) against the
    oracle, and the autotuner's per-shape cache: dg_autotune stores its
    choice, a new handle of the same shape takes it with dg_tune_lookup, and
    the JSON file written by dg_tune_cache_save holds it."""
    import json
    from diablo_b200 import _lib
    p, gy = configs.kh_shear_layer(nx=128, ny=33, nz=32)
    ref, ch, _ = start_pair(p, gy, ics.kh_shear_layer, seed=5)
    ch.tune_set(fft_plan=1)
    for s in range(1, 21):
        ref.step(s)
        ch.step(s)
    compare(ref, ch, fields(p))
    ch.set_state(ref.state())
    tuned = ch.autotune(1)
    ch.close()
    other = channel(p, gy)
    assert other.tune_lookup()
    assert other.tune_get() == tuned
    other.close()
    path = tmp_path / "tune.json"
    _lib.tune_cache_save(str(path))
    key = f"{p.nx}x{p.ny}x{p.nz}_th{p.n_th}_fp64"
    assert json.loads(path.read_text())[key] == {k: tuned[k] for k in
                                                 ("col_mt", "xrow_chunk", "ychunk", "cn_mt",
                                                  "pdl", "fft_plan")}


@pytest.mark.parametrize("case", ["coupled", "uncoupled"])
@pytest.mark.parametrize("mt", [2, 4, 16])
def test_column_stage_tiles_match_oracle(case, mt):
    """The column stage at small and large tiles (DG_TUNE_CN_MT) against the
    oracle, with COURANT every step (substep 3 runs COURANT on the post-CN
    velocity before the projection).  "coupled": a stratified KH layer with
    rotation, gravity in x and z, and a Neumann scalar with DRHODX/Z -- every
    field's right-hand side reads others, and both scalars go through the
    rhs arrays; "uncoupled": a small no-slip channel with a passive scalar
    written in place."""
    if case == "coupled":
        p, gy = configs.kh_shear_layer(nx=32, ny=33, nz=16)
        p = p.replace(i_ro=0.3, grav_x=0.2, grav_z=-0.1, variable_dt=1, update_dt=1, cfl=0.4,
                      n_th=2)
        p.ri = [0.1, 0.05, 0, 0]
        p.pr = [1.0, 0.7, 1, 1]
        p.th_bc_ymin = [0, 1, 0, 0]
        p.th_bc_ymax = [0, 1, 0, 0]
        p.th_bc_ymin_c1 = [-1.0, 0.1, 0, 0]
        p.th_bc_ymax_c1 = [1.0, -0.2, 0, 0]
        p.drhodx = [0.0, 0.3, 0, 0]
        p.drhodz = [0.0, -0.2, 0, 0]
        maker = ics.kh_shear_layer
    else:
        p, gy = configs.channel_re180(nx=48, ny=33, nz=32)
        p = p.replace(n_th=1)
        p.pr = [0.71, 1, 1, 1]
        p.ri = [0.0, 0, 0, 0]
        p.th_bc_ymin = [0, 0, 0, 0]
        p.th_bc_ymax = [0, 0, 0, 0]
        p.th_bc_ymin_c1 = [-1.0, 0, 0, 0]
        p.th_bc_ymax_c1 = [1.0, 0, 0, 0]
        maker = ics.channel_laminar
    ref, ch, _ = start_pair(p, gy, maker, seed=12)
    ch.tune_set(cn_mt=mt)
    for s in range(1, 11):
        ref.step(s)
        ch.step(s)
    compare(ref, ch, fields(p) + ["CP"], tol=1e-10)
    t_o, dt_o = ref.get_time()
    t_g, dt_g = ch.get_time()
    assert abs(dt_g - dt_o) <= 1e-12 * dt_o
    ch.close()
