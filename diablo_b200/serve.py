"""Python mirror of the ensemble server (dg_server_* in include/diablo_b200.h):
continuous batching of independent channel solves on one GPU."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import DgParams, Params


class ServerStats(ctypes.Structure):
    _fields_ = [("cases_done", ctypes.c_int64), ("steps_done", ctypes.c_int64),
                ("active", ctypes.c_int32), ("queued", ctypes.c_int32),
                ("bytes_active", ctypes.c_int64), ("bytes_peak", ctypes.c_int64),
                ("step_ms_p50", ctypes.c_double), ("step_ms_p99", ctypes.c_double),
                ("cases_per_s", ctypes.c_double), ("mpoint_steps_per_s", ctypes.c_double),
                ("wall_s", ctypes.c_double)]


def state_names(p: Params):
    return ["CU1", "CU2", "CU3", "CP"] + [f"CTH{n}" for n in range(p.n_th)]


def state_bytes(p: Params) -> int:
    """Device bytes a handle for `p` allocates (dg_state_bytes)."""
    L = _lib.load()
    return int(L.dg_state_bytes(ctypes.byref(p.to_struct(DgParams))))


class Server:
    def __init__(self, max_active: int = 32, budget_gb: float = 150.0, autotune: bool = True):
        self.L = _lib.load()
        s = ctypes.c_void_p()
        _lib.check("dg_server_create",
                   self.L.dg_server_create(max_active, float(budget_gb), int(autotune),
                                           ctypes.byref(s)))
        self.s = s
        self._params = {}

    def submit(self, p: Params, gy: np.ndarray, state: dict, nsteps: int,
               prepare: bool = True) -> int:
        """Queue one case.  state: compact spectral CU1, CU2, CU3, CP, CTHn
        ([NY+2][TNKZ+1][NKX+1] complex); prepare applies APPLY_BC_VEL,
        REM_DIV_CHAN, APPLY_BC_VEL on admission."""
        names = state_names(p)
        arrs = [np.ascontiguousarray(state[n], dtype=np.complex128) for n in names]
        ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        g = np.ascontiguousarray(gy, dtype=np.float64)
        cid = ctypes.c_int64()
        _lib.check("dg_server_submit",
                   self.L.dg_server_submit(self.s, ctypes.byref(p.to_struct(DgParams)),
                                           g.ctypes.data_as(ctypes.c_void_p), ptrs, int(nsteps),
                                           int(prepare), ctypes.byref(cid)))
        self._params[cid.value] = p
        return cid.value

    def wait(self, cid: int):
        """Block until the case is done; returns (state dict, (queued_s, run_s))."""
        p = self._params.pop(cid)
        names = state_names(p)
        outs = [np.zeros(p.spec_shape(), dtype=np.complex128) for _ in names]
        ptrs = (ctypes.c_void_p * len(outs))(*[a.ctypes.data for a in outs])
        times = (ctypes.c_double * 2)()
        _lib.check("dg_server_wait", self.L.dg_server_wait(self.s, int(cid), ptrs, times))
        return dict(zip(names, outs)), (times[0], times[1])

    def stats(self) -> dict:
        st = ServerStats()
        _lib.check("dg_server_query", self.L.dg_server_query(self.s, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "s", None):
            self.L.dg_server_destroy(self.s)
            self.s = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
