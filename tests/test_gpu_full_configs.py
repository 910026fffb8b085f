"""The two largest workload configurations at their stated sizes and lengths,
FP64 and mixed precision, both against the FP64 oracle (needs a B200).

* Triply periodic decaying turbulence, 256^3, nu = 1e-3, seeded
  k^4 exp(-2 (k/4)^2) spectrum, 200 RK3 steps (RK_PER_1,
  for/periodic.f:23-285): FP64 within 1e-11 relative L2 per field, mixed
  within 1e-5, divergence at the FP64 level for both, KE series every 50
  steps.
* Channel at Re_tau ~ 550, 512 x 257 x 384 with one passive scalar, COURANT
  every step (RK_CHAN_1, for/channel.f:62-1073): the oracle needs 10-25 s of
  the host's cores per step at this size, so the comparison runs the first
  10 steps from the seeded state: FP64 within 1e-11, mixed within 1e-5,
  DELTA_T and TIME, max |div u|.  (The mixed form is also compared with the
  FP64 GPU path over 100 steps in test_gpu_mixed.py.)

The oracle advances once; the FP64 and the mixed GPU runs start from its
state and step beside it.  Each test prints its per-field errors
(pytest -s shows them).
"""
import json

import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics

pytestmark = pytest.mark.gpu

TOL = 1e-11
TOL_MIXED = 1e-5


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def fields(p):
    return ["CU1", "CU2", "CU3"] + [f"CTH{n}" for n in range(p.n_th)]


def report(name, rec):
    print(f"\nPARITY {name} " + json.dumps(rec, sort_keys=True))


def test_periodic_256_cubed_200_steps_fp64_and_mixed():
    from diablo_b200.solver import Periodic
    p, _ = configs.periodic_256()
    ref = O.Oracle(p, None)
    for nm, a in zip(("CU1", "CU2", "CU3"), ics.periodic_spectrum(p, seed=3)):
        ref.set(nm, a)
    ref.rem_div_per()
    ref.poisson_p_per()
    start = ref.state()
    runs = {}
    for prec in (0, 1):
        g = Periodic(p.replace(precision=prec))
        g.set_state(start)
        g.set_time(0.0, p.delta_t)
        runs[prec] = g
    ke = {0: [], 1: [], "oracle": []}
    for s in range(1, 201):
        ref.step(s)
        for g in runs.values():
            g.steps(s, 1)
        if s % 50 == 0:
            ke["oracle"].append(ref.stats()["ke"])
            for prec, g in runs.items():
                st = g.stats()
                ke[prec].append(st["ke"])
                assert st["div_max"] <= 1e-12 * 256, (s, prec, st["div_max"])
    out = {}
    for prec, g in runs.items():
        err = {nm: rel(g.get_field(nm), ref.get(nm)) for nm in fields(p)}
        ke_err = max(abs(a - b) / b for a, b in zip(ke[prec], ke["oracle"]))
        out["mixed" if prec else "fp64"] = {"rel_l2": err, "ke_rel_err_max": ke_err,
                                            "div_max": g.stats()["div_max"]}
    report("periodic_256cubed_200_steps", out)
    assert all(v <= TOL for v in out["fp64"]["rel_l2"].values()), out
    assert out["fp64"]["ke_rel_err_max"] <= 1e-12, out
    assert all(v <= TOL_MIXED for v in out["mixed"]["rel_l2"].values()), out
    assert out["mixed"]["ke_rel_err_max"] <= 1e-6, out
    t_o, _ = ref.get_time()
    for g in runs.values():
        assert abs(g.get_time()[0] - t_o) <= 1e-12 * t_o
        g.close()
    ref.close()


def test_channel_re550_full_grid_fp64_and_mixed():
    from diablo_b200.solver import Channel
    p, gy = configs.channel_re550()
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = ics.channel_laminar(p, gy, seed=4)
    ref.create_flow_chan(u1, u2, u3, th)
    start = ref.state()
    runs = {}
    for prec in (0, 1):
        g = Channel(p.replace(precision=prec), gy)
        g.set_state(start)
        g.set_time(0.0, p.delta_t)
        runs[prec] = g
    nsteps = 10
    for s in range(1, nsteps + 1):
        ref.step(s)
        for g in runs.values():
            g.steps(s, 1)
    t_o, dt_o = ref.get_time()
    so = ref.stats()
    out = {}
    for prec, g in runs.items():
        err = {nm: rel(g.get_field(nm), ref.get(nm)) for nm in fields(p)}
        t_g, dt_g = g.get_time()
        sg = g.stats()
        out["mixed" if prec else "fp64"] = {
            "rel_l2": err, "delta_t_rel_err": abs(dt_g - dt_o) / dt_o,
            "time_rel_err": abs(t_g - t_o) / t_o, "div_max": sg["div_max"],
            "ke_rel_err": abs(sg["ke"] - so["ke"]) / so["ke"]}
    report(f"channel_re550_512x257x384_{nsteps}_steps", out)
    f64, mx = out["fp64"], out["mixed"]
    assert all(v <= TOL for v in f64["rel_l2"].values()), out
    assert f64["delta_t_rel_err"] <= 1e-12 and f64["time_rel_err"] <= 1e-12, out
    assert f64["div_max"] <= 1e-12 and f64["ke_rel_err"] <= 1e-12, out
    assert all(v <= TOL_MIXED for v in mx["rel_l2"].values()), out
    assert mx["delta_t_rel_err"] <= 1e-6 and mx["div_max"] <= 1e-12, out
    for g in runs.values():
        g.close()
    ref.close()
