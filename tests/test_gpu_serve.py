"""The continuous-batching ensemble server (needs a B200): each result is the
same alone and in the mix, admission respects slots and the HBM budget, and
a failing request does not stop the others."""
import numpy as np
import pytest

from diablo_b200 import configs, ics
from diablo_b200.serve import Server, state_bytes, state_names

pytestmark = pytest.mark.gpu


def cases():
    """Six small KH cases of different sizes and physics, FP64 and mixed."""
    out = []
    shapes = [(32, 17, 16), (64, 33, 16), (48, 17, 32), (64, 17, 32), (32, 33, 16), (96, 17, 16)]
    for i, (nx, ny, nz) in enumerate(shapes):
        p, gy = configs.kh_shear_layer(nx=nx, ny=ny, nz=nz)
        p = p.replace(nu=1.0 / (600 + 500 * i), precision=i % 2)
        p.ri = [0.05 + 0.03 * i, 0, 0, 0]
        out.append((p, gy, ics.kh_state(p, gy, seed=20 + i), 15 + 3 * i))
    return out


def alone(p, gy, st, nsteps):
    """The case on its own handle, with the launch shapes the server's
    autotuner stored for its grid shape (the transform plan variant changes
    results at round-off level, so both sides must use the same one)."""
    from diablo_b200.solver import Channel
    ch = Channel(p, gy)
    ch.tune_lookup()
    for k, v in st.items():
        ch.set_field(k, v)
    ch.set_time(0.0, p.delta_t)
    ch.apply_bc_vel()
    ch.rem_div_chan()
    ch.apply_bc_vel()
    ch.steps(1, nsteps)
    res = {n: ch.get_field(n) for n in state_names(p)}
    ch.close()
    return res


def courant_cases():
    """Small no-slip channels with variable DELTA_T: COURANT every step (can
    join a group: the column launch of substep 3 stops after its CN solves)
    and every other step (steps alone in grouped mode)."""
    out = []
    for i, upd in enumerate((1, 2)):
        p, gy = configs.channel_re180(nx=32, ny=17, nz=32)
        p = p.replace(update_dt=upd, precision=i)
        u1, u2, u3, _ = ics.channel_laminar(p, gy, seed=40 + i)
        from diablo_b200.solver import Channel
        ch = Channel(p, gy)
        ch.create_flow(u1, u2, u3)
        st = {n: ch.get_field(n) for n in state_names(p)}
        ch.close()
        out.append((p, gy, st, 12))
    return out


@pytest.mark.parametrize("group", [0, 3])
def test_each_result_same_alone_and_in_the_mix(group):
    """group = 0: every case steps on its own stream; group = 3: cases of
    similar size step together, one ragged column launch per substep."""
    cs = cases() + courant_cases()
    with Server(max_active=5, budget_gb=0, autotune=True, group_cases=group) as srv:
        ids = [srv.submit(p, gy, st, n) for p, gy, st, n in cs]
        res = [srv.wait(i) for i in ids]
        s = srv.stats()
    solo = [alone(*c) for c in cs]
    for (got, times), want, c in zip(res, solo, cs):
        for nm in want:
            assert np.array_equal(got[nm], want[nm]), (c[0].nx, c[0].ny, c[0].nz, nm)
    assert s["cases_done"] == len(cs)
    assert s["steps_done"] == sum(c[3] for c in cs)
    assert 0 < s["step_ms_p50"] <= s["step_ms_p99"]


def test_budget_admission_and_errors():
    cs = cases()[:4]
    # room for the two largest cases at most
    budget = sorted(state_bytes(c[0]) for c in cs)[-1] * 2.05 / 1e9
    bad = cs[0][0].replace(nx=28)               # NX with a factor of 7: refused
    with Server(max_active=8, budget_gb=budget, autotune=False) as srv:
        ids = [srv.submit(p, gy, st, 5) for p, gy, st, _ in cs]
        bad_id = srv.submit(bad, cs[0][1], cs[0][2], 5)
        for i in ids:
            srv.wait(i)
        with pytest.raises(Exception) as e:
            srv.wait(bad_id)
        assert getattr(e.value, "code", None) == 2
        s = srv.stats()
    assert s["cases_done"] == len(cs)
    assert s["bytes_peak"] <= budget * 1e9
