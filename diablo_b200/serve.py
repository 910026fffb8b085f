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
    def __init__(self, max_active: int = 32, budget_gb: float = 150.0, autotune: bool = True,
                 group_cases: int = 0):
        """group_cases > 0: cases of similar size step together in groups of
        up to that many, one graph per group step with one ragged column
        launch per substep (dg_server_config DG_SERVER_GROUP_CASES)."""
        self.L = _lib.load()
        s = ctypes.c_void_p()
        _lib.check("dg_server_create",
                   self.L.dg_server_create(max_active, float(budget_gb), int(autotune),
                                           ctypes.byref(s)))
        self.s = s
        self._params = {}
        if group_cases:
            _lib.check("dg_server_config", self.L.dg_server_config(self.s, 0, int(group_cases)))

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


# ------------------------------------------------------------ several GPUs
# The ensemble shards as independent units: every case runs whole on one GPU
# (one server per GPU, one process per GPU), so no data crosses between GPUs
# and there is no collective on the data path.  A host-side dispatcher
# assigns the cases; the ranks exchange only their statistics at the end.

def assign_cases(work, world: int):
    """Rank of each case: longest-processing-time first, each case to the
    least-loaded rank so far (ties to the lower rank).  `work` is any
    per-case cost, e.g. points x steps.  Deterministic, so every rank
    computes the same assignment without communicating."""
    work = [float(w) for w in work]
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    load = [0.0] * world
    rank_of = [0] * len(work)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        rank_of[i] = r
        load[r] += work[i]
    return rank_of


def merge_rank_stats(per_rank):
    """Whole-job ensemble figures from each rank's record: points and cases
    summed, divided by the slowest rank's wall time (the job lasts as long
    as its slowest GPU); case latencies pooled for exact percentiles; step
    latency percentiles as the worst rank's (the servers keep no samples)."""
    wall = max(r["wall_s"] for r in per_rank)
    pts = sum(r["points"] for r in per_rank)
    cases = sum(r["cases"] for r in per_rank)
    lat = [x for r in per_rank for x in r["case_latency_s"]]
    return {"ranks": len(per_rank), "cases": cases, "wall_s": wall,
            "cases_per_s": cases / wall if wall > 0 else 0.0,
            "mpoint_steps_per_s": pts / wall / 1e6 if wall > 0 else 0.0,
            "step_ms_p50_worst_rank": max(r["step_ms_p50"] for r in per_rank),
            "step_ms_p99_worst_rank": max(r["step_ms_p99"] for r in per_rank),
            "case_latency_s_p50": float(np.percentile(lat, 50)) if lat else 0.0,
            "case_latency_s_p99": float(np.percentile(lat, 99)) if lat else 0.0,
            "hbm_peak_gb_max": max(r["hbm_peak_gb"] for r in per_rank)}
