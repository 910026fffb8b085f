"""Parity of the sm_100a triply periodic path (RK_PER_1, REM_DIV_PER,
POISSON_P_PER, FFT_XZY_*) with the CPU oracle (needs a B200).

Tolerances as for the channel: relative L2 <= 1e-11 on the prognostic fields
after the stated number of steps, max |div u| <= 1e-12 (scaled by the
velocity gradient for the large cases), matching KE series.
"""
import math

import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics
from diablo_b200.params import Params

pytestmark = pytest.mark.gpu

TOL = 1e-11


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def periodic(p):
    from diablo_b200.solver import Periodic
    return Periodic(p)


def box(n=(32, 32, 32), **kw):
    nx, ny, nz = n
    q = dict(nx=nx, ny=ny, nz=nz, num_per_dir=3, nu=0.01, lx=2 * math.pi, ly=2 * math.pi,
             lz=2 * math.pi, delta_t=0.005, variable_dt=0)
    q.update(kw)
    return Params(**q)


def seeded_pair(p, seed=3, scalars=None):
    """Oracle and GPU solver holding the same divergence-free state: the
    seeded random spectrum, REM_DIV_PER and POISSON_P_PER on the oracle, the
    resulting state copied to the device."""
    ref = O.Oracle(p, None)
    for nm, a in zip(("CU1", "CU2", "CU3"), ics.periodic_spectrum(p, seed=seed)):
        ref.set(nm, a)
    for n in range(p.n_th):
        th = ics.periodic_spectrum(p, seed=seed + 10 + n)[0]
        if scalars is not None:
            th = th * scalars[n]
        ref.set(f"CTH{n}", th)
    ref.rem_div_per()
    ref.poisson_p_per()
    g = periodic(p)
    g.set_state(ref.state())
    g.set_time(0.0, p.delta_t)
    return ref, g


def fields(p):
    return ["CU1", "CU2", "CU3"] + [f"CTH{n}" for n in range(p.n_th)]


@pytest.mark.parametrize("n", [(32, 32, 32), (48, 24, 96), (64, 16, 128), (36, 18, 24),
                               (256, 256, 16)])
def test_fft_xzy_matches_oracle(n):
    p = box(n)
    ref = O.Oracle(p, None)
    g = periodic(p)
    rng = np.random.default_rng(sum(n))
    phys = rng.standard_normal(p.phys_shape())
    spec = ref.to_fourier(phys)
    assert rel(g.to_fourier(phys), spec) < 1e-14
    assert rel(g.to_physical(spec), ref.to_physical(spec)) < 1e-14
    # reference layout: the retained block, zeros elsewhere; aliased in place
    U = np.zeros((p.ny + 2, p.nz + 2, p.nx + 2))
    U[: p.ny, : p.nz, : p.nx] = phys
    CU = U.view(np.complex128)                     # same memory, CU(0:NX/2,0:NZ+1,0:NY+1)
    g.fft_xzy_to_fourier(U, CU)
    blk = CU[: p.tnky + 1, : p.tnkz + 1, : p.nkx + 1]
    assert rel(blk, spec) < 1e-14
    assert np.all(CU[p.tnky + 1:] == 0) and np.all(CU[:, :, p.nkx + 1:] == 0)
    g.fft_xzy_to_physical(CU, U)
    assert rel(U[: p.ny, : p.nz, : p.nx], ref.to_physical(spec)) < 1e-14
    g.close()


def test_rem_div_and_poisson_match_oracle():
    p = box((64, 64, 64))
    ref = O.Oracle(p, None)
    rng = np.random.default_rng(7)
    # a field that is NOT divergence-free, so the projection does work
    u = [rng.standard_normal(p.phys_shape()) for _ in range(3)]
    g = periodic(p)
    for nm, a in zip(("CU1", "CU2", "CU3"), u):
        ref.set(nm, ref.to_fourier(a))
        g.set_field(nm, ref.get(nm))
    ref.rem_div_per()
    g.rem_div_per()
    for nm in ("CU1", "CU2", "CU3", "CR1"):
        assert rel(g.get_field(nm), ref.get(nm)) < 1e-13, nm
    # REM_DIV_PER divides by k^2 + EPS (EPS ~ 1e-9), so the lowest modes keep
    # EPS/k^2 of their divergence in the reference too
    dg, do = g.stats()["div_max"], ref.div_max()
    assert abs(dg - do) <= 1e-6 * do + 1e-13
    ref.poisson_p_per()
    g.poisson_p_per()
    assert rel(g.get_field("CP"), ref.get("CP")) < 1e-12
    g.close()


def test_create_flow_matches_oracle():
    p = box((32, 48, 32))
    rng = np.random.default_rng(8)
    u = [rng.standard_normal(p.phys_shape()) for _ in range(3)]
    ref = O.Oracle(p, None)
    ref.create_flow_per(*u)
    g = periodic(p)
    g.create_flow(*u)
    for nm in ("CU1", "CU2", "CU3", "CP"):
        assert rel(g.get_field(nm), ref.get(nm)) < 1e-12, nm
    g.close()


def test_shear_mode_decays_exactly():
    """u1 = sin(y): no nonlinear transfer, each substep multiplies the mode by
    (1 - nu h k^2/2)/(1 + nu h k^2/2)."""
    n = 32
    p = box((n, n, n), nu=0.05, delta_t=0.01)
    g = periodic(p)
    y = np.arange(n) * 2 * math.pi / n
    u1 = np.sin(y)[:, None, None] * np.ones((n, n, n))
    z = np.zeros((n, n, n))
    g.create_flow(u1, z, z)
    a0 = g.get_field("CU1")[1, 0, 0]
    for s in range(10):
        g.step(s + 1)
    amp = 1.0
    for _ in range(10):
        for h in (8 / 15, 2 / 15, 5 / 15):
            t = p.nu * h * p.delta_t / 2
            amp *= (1 - t) / (1 + t)
    c = g.get_field("CU1")
    assert abs(c[1, 0, 0] - a0 * amp) < 1e-14
    c[1, 0, 0] = c[-1, 0, 0] = 0
    assert np.abs(c).max() < 1e-15
    g.close()


def test_decaying_64_cubed_100_steps():
    p = box((64, 64, 64), nu=5e-3, delta_t=4e-3)
    ref, g = seeded_pair(p)
    for s in range(1, 101):
        ref.step(s)
        g.step(s)
        if s % 20 == 0:
            so, sg = ref.stats(), g.stats()
            assert abs(sg["ke"] - so["ke"]) <= 1e-12 * so["ke"]
            assert sg["div_max"] <= 1e-12 * 64
    for nm in fields(p) + ["CP"]:
        assert rel(g.get_field(nm), ref.get(nm)) <= TOL, nm
    t_o, _ = ref.get_time()
    t_g, _ = g.get_time()
    assert abs(t_g - t_o) < 1e-12
    g.close()


@pytest.mark.parametrize("variant", ["one_scalar_bg", "two_scalars_forced", "generic_x",
                                     "three_scalars"])
def test_periodic_variants(variant):
    if variant == "one_scalar_bg":
        p = box((32, 32, 32), n_th=1)
        p.ri = [0.3, 0, 0, 0]
        p.pr = [0.7, 1, 1, 1]
        p.background_grad = [1, 0, 0, 0]
    elif variant == "two_scalars_forced":
        p = box((48, 32, 16), n_th=2, epsilon_target=0.2)
        p.ri = [0.2, -0.1, 0, 0]
        p.pr = [1.0, 2.0, 1, 1]
        p.background_grad = [0, 1, 0, 0]
    elif variant == "generic_x":            # NX without a warp specialisation
        p = box((36, 24, 18), n_th=1)
        p.ri = [0.1, 0, 0, 0]
        p.pr = [1.0, 1, 1, 1]
    else:                                   # N_TH = 3: generic product path
        p = box((32, 16, 32), n_th=3)
        p.ri = [0.1, 0.05, 0.02, 0]
        p.pr = [1.0, 0.5, 2.0, 1]
        p.background_grad = [1, 0, 1, 0]
    ref, g = seeded_pair(p, seed=5, scalars=[0.5] * p.n_th)
    for s in range(1, 11):
        ref.step(s)
        g.step(s)
    for nm in fields(p) + ["CF1", "CF2", "CF3", "CP"]:
        assert rel(g.get_field(nm), ref.get(nm)) <= 1e-10, nm
    so, sg = ref.stats(), g.stats()
    for n in range(p.n_th):
        assert abs(sg["th_var"][n] - so["th_var"][n]) <= 1e-10 * so["th_var"][n]
    g.close()


def test_graph_steps_match_substep_calls():
    p = box((32, 32, 32), n_th=1)
    p.ri = [0.2, 0, 0, 0]
    ref, a = seeded_pair(p, seed=9, scalars=[0.5])
    b = periodic(p)
    b.set_state(ref.state())
    b.set_time(0.0, p.delta_t)
    for s in range(1, 9):
        a.step(s)
    b.steps(1, 8)
    for nm in fields(p) + ["CP"]:
        assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
    a.close()
    b.close()
