"""The bounded wait of the bulk-copy (TMA) column staging, made to run out
without any fault (needs a B200).

The Crank-Nicolson column kernel stages its right-hand-side tile with bulk
tensor copies completed on an mbarrier and polls the barrier a bounded number
of times.  The test knob (DG_TUNE_WAIT_TEST) lowers the poll limit for one
launch and makes the barrier expect 16 bytes more than the copies bring: every
copy lands in the CTA's own shared memory, the barrier simply never completes,
and the wait gives up.  The kernel must flag the failure and skip its work,
diablo_synchronize must report DG_ERR_TIMEOUT once, and the handle must stay
usable: the next normal step matches the oracle.
"""
import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics
from diablo_b200._lib import DiabloError

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_wait_limit_reports_timeout_and_handle_recovers():
    from diablo_b200.solver import Channel
    p, gy = configs.kh_shear_layer(nx=32, ny=17, nz=16)
    u1, u2, u3, th = ics.kh_shear_layer(p, gy, seed=11, kick=1e-2)
    ref = O.Oracle(p, gy)
    ref.create_flow_chan(u1, u2, u3, th)
    start = ref.state()
    ch = Channel(p, gy)
    ch.set_state(start)
    ch.set_time(0.0, p.delta_t)
    ch.synchronize()  # nothing pending before the test

    ch.wait_test(64)
    for rk in (1, 2, 3):
        ch.rk_chan_1(1, rk)           # substep 1's CN launch gives up; the rest run normally
    with pytest.raises(DiabloError) as exc:
        ch.synchronize()
    assert exc.value.code == 6, exc.value          # DG_ERR_TIMEOUT
    assert "wait limit" in str(exc.value)
    ch.synchronize()                               # reported once, then clear

    # the same handle, restarted from the oracle's state, steps correctly
    ch.set_state(start)
    ch.set_time(0.0, p.delta_t)
    ref.step(1)
    ch.step(1)
    ch.synchronize()
    for k in ("CU1", "CU2", "CU3", "CTH0"):
        assert rel(ch.get_field(k), ref.get(k)) < 1e-12, k
    ch.close()
