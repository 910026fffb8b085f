"""Host-side mirror of the reference's stepper interface.

``Channel`` and ``Periodic`` wrap one device handle and expose the
reference's subroutines under their own names (``rk_chan_1``,
``rem_div_chan``, ``fft_xz_to_fourier`` ...), with the same argument meaning,
so a driver loop reads like ``for/diablo.f:66-120``::

    for time_step in range(1, n + 1):
        for rk_step in (1, 2, 3):
            ch.rk_chan_1(time_step, rk_step)
        ch.advance_time()          # TIME = TIME + DELTA_T

Errors raise ``DiabloError`` (the reference would ``STOP``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .grid import grid_metrics
from .params import DgParams, Params

__all__ = ["Channel", "Periodic", "DiabloError"]

DiabloError = _lib.DiabloError


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _cstrings(paths, n):
    if not paths:
        return None
    arr = (ctypes.c_char_p * max(n, 1))()
    for i in range(n):
        arr[i] = paths[i].encode() if i < len(paths) and paths[i] else None
    return arr


class _Solver:
    def __init__(self, p: Params, gy=None, stream=None):
        self.L = _lib.load()
        self.p = p
        self._dp = p.to_struct(DgParams)
        self._gy = None if gy is None else np.ascontiguousarray(gy, dtype=np.float64)
        h = ctypes.c_void_p()
        code = self.L.diablo_gpu_init(ctypes.byref(self._dp),
                                      None if self._gy is None else _ptr(self._gy),
                                      None if stream is None else ctypes.c_void_p(stream),
                                      ctypes.byref(h))
        _lib.check("diablo_gpu_init", code)
        self.h = h
        self.spec_shape = p.spec_shape()
        self.phys_shape = p.phys_shape()

    def close(self):
        if getattr(self, "h", None):
            self.L.diablo_gpu_finalize(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args):
        _lib.check(name, getattr(self.L, name)(self.h, *args))

    TUNE_KEYS = {"col_mt": 0, "xrow_chunk": 1, "ychunk": 2, "cn_mt": 3, "pdl": 4, "fft_plan": 6,
                 "plane_xz": 7}

    def tune_set(self, **kw):
        """Launch-shape tunables (results do not depend on them)."""
        for k, v in kw.items():
            self._call("dg_tune_set", self.TUNE_KEYS[k], int(v))

    def tune_get(self) -> dict:
        out = {}
        for k, key in self.TUNE_KEYS.items():
            v = ctypes.c_int()
            self._call("dg_tune_get", key, ctypes.byref(v))
            out[k] = v.value
        return out

    def wait_test(self, polls: int):
        """Test only: the next Crank-Nicolson column launch gives up on its
        bulk-copy barrier after `polls` polls (its copies all land; the
        barrier expects 16 bytes more), skips its work and flags the failure,
        which the next synchronize / stats call reports once as
        DG_ERR_TIMEOUT."""
        self._call("dg_tune_set", 5, int(polls))

    def autotune(self, steps_per_trial: int = 3) -> dict:
        """Time candidate launch shapes on this state, keep the fastest; the
        state, TIME and DELTA_T are restored afterwards.  The choice also goes
        into the process-wide tuning cache (tune_cache_save / _load)."""
        self._call("dg_autotune", steps_per_trial)
        return self.tune_get()

    def tune_lookup(self) -> bool:
        """Apply the tuning cache's entry for this grid shape, if any."""
        hit = ctypes.c_int()
        self._call("dg_tune_lookup", ctypes.byref(hit))
        return bool(hit.value)

    def steps(self, time_step: int, nsteps: int):
        """nsteps full RK3 steps from time_step (the driver loop body,
        for/diablo.f:70-109), replayed as CUDA graphs after the first."""
        self._call("diablo_step", time_step, nsteps)

    # ---- state I/O
    _LAYOUTS = {"compact": _lib.DG_LAYOUT_COMPACT, "reference": _lib.DG_LAYOUT_REFERENCE,
                "reference_retained": _lib.DG_LAYOUT_REFERENCE_RETAINED}

    def set_field(self, name: str, arr: np.ndarray, layout: str = "compact"):
        a = np.ascontiguousarray(arr, dtype=np.complex128)
        lay = self._LAYOUTS[layout]
        if lay == _lib.DG_LAYOUT_COMPACT and a.size != int(np.prod(self.spec_shape)):
            raise ValueError(f"{name}: expected {self.spec_shape}, got {a.shape}")
        self._call("diablo_set_field", _lib.field_id(name), _ptr(a), lay, _lib.DG_HOST)

    def get_field(self, name: str, layout: str = "compact", out: np.ndarray | None = None):
        """A spectral field in the compact or the reference layout.  With
        "reference_retained" only the retained block of `out` is written (the
        rest keeps its contents; a new array starts at zero)."""
        lay = self._LAYOUTS[layout]
        if lay == _lib.DG_LAYOUT_COMPACT:
            shp = self.spec_shape
        else:
            shp = (self.spec_shape[0], self.p.nz + 2, self.p.nx // 2 + 1)
        if out is None:
            out = np.zeros(shp, dtype=np.complex128)
        elif out.shape != shp or out.dtype != np.complex128 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"{name}: out must be a contiguous complex128 array of {shp}")
        self._call("diablo_get_field", _lib.field_id(name), _ptr(out), lay, _lib.DG_HOST)
        return out

    def set_fields(self, arrays: dict, layout: str = "compact"):
        """Several fields in one call (diablo_set_fields: two copy streams, one
        synchronisation)."""
        names = list(arrays)
        lay = self._LAYOUTS[layout]
        arrs = [np.ascontiguousarray(arrays[n], dtype=np.complex128) for n in names]
        ids = (ctypes.c_int * len(names))(*[_lib.field_id(n) for n in names])
        ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        self._call("diablo_set_fields", len(names), ids, ptrs, lay, _lib.DG_HOST)

    def get_fields(self, out: dict, layout: str = "compact"):
        """Fill the arrays of `out` (name -> contiguous complex128 array of the
        layout's shape) in one call (diablo_get_fields)."""
        names = list(out)
        for n in names:
            a = out[n]
            if a.dtype != np.complex128 or not a.flags["C_CONTIGUOUS"]:
                raise ValueError(f"{n}: out arrays must be contiguous complex128")
        ids = (ctypes.c_int * len(names))(*[_lib.field_id(n) for n in names])
        ptrs = (ctypes.c_void_p * len(names))(*[out[n].ctypes.data for n in names])
        self._call("diablo_get_fields", len(names), ids, ptrs, self._LAYOUTS[layout], _lib.DG_HOST)
        return out

    def set_field_device(self, name: str, dev_ptr: int):
        """Copy a compact-layout complex128 field from device memory."""
        self._call("diablo_set_field", _lib.field_id(name), ctypes.c_void_p(dev_ptr),
                   _lib.DG_LAYOUT_COMPACT, _lib.DG_DEVICE)

    def get_field_device(self, name: str, dev_ptr: int):
        self._call("diablo_get_field", _lib.field_id(name), ctypes.c_void_p(dev_ptr),
                   _lib.DG_LAYOUT_COMPACT, _lib.DG_DEVICE)

    def save_flow(self, path: str, time_step: int, th_paths=None):
        """SAVE_FLOW without HDF5 (for/diablo_io.f:307-404)."""
        arr = _cstrings(th_paths, self.p.n_th)
        self._call("diablo_save_flow", int(time_step), path.encode(), arr)

    def read_flow(self, path: str, th_paths=None) -> int:
        """READ_FLOW without HDF5 (for/diablo_io.f:201-305); returns
        TIME_STEP and sets TIME from the file."""
        arr = _cstrings(th_paths, self.p.n_th)
        ts = ctypes.c_int()
        self._call("diablo_read_flow", path.encode(), arr, ctypes.byref(ts))
        return ts.value

    def state_names(self):
        n = ["CU1", "CU2", "CU3", "CP", "CF1", "CF2", "CF3"]
        n += [f"CTH{k}" for k in range(self.p.n_th)] + [f"CFTH{k}" for k in range(self.p.n_th)]
        return n

    def get_state(self) -> dict:
        return {k: self.get_field(k) for k in self.state_names()}

    def set_state(self, st: dict):
        for k, v in st.items():
            self.set_field(k, v)

    def set_time(self, time: float, delta_t: float):
        self._call("diablo_set_time", ctypes.c_double(time), ctypes.c_double(delta_t))

    def get_time(self):
        t, d = ctypes.c_double(), ctypes.c_double()
        self._call("diablo_get_time", ctypes.byref(t), ctypes.byref(d))
        return t.value, d.value

    def advance_time(self):
        self._call("diablo_advance_time")

    def synchronize(self):
        self._call("diablo_synchronize")

    def stats(self) -> dict:
        s = _lib.DgStats()
        self._call("diablo_stats", ctypes.byref(s))
        d = {k: getattr(s, k) for k in ("ubulk", "urms_b", "vrms_b", "wrms_b", "ke", "div_max")}
        d["thrms_b"] = list(s.thrms_b)[: self.p.n_th]
        d["th_var"] = list(s.th_var)[: self.p.n_th]
        return d


class Channel(_Solver):
    """Device-resident channel state driven through RK_CHAN_1 and helpers."""

    def flow_fields_physical(self, pressure: bool = True) -> dict:
        """The datasets of the reference's HDF5 flow file (WriteHDF5,
        for/hdf5.f:5-292): physical U, V (on GYF), W, TH<n> and P on planes
        1..NY as [NZ][NY][NX] arrays."""
        nz, ny, nx = self.p.nz, self.p.ny, self.p.nx
        U, V, W = (np.zeros((nz, ny, nx)) for _ in range(3))
        TH = np.zeros((max(self.p.n_th, 1), nz, ny, nx))
        P = np.zeros((nz, ny, nx)) if pressure else None
        self._call("diablo_flow_fields_physical", _ptr(U), _ptr(V), _ptr(W),
                   _ptr(TH) if self.p.n_th else None, _ptr(P) if pressure else None)
        out = {"U": U, "V": V, "W": W}
        for n in range(self.p.n_th):
            out[f"TH{n + 1}"] = TH[n]
        if pressure:
            out["P"] = P
        return out

    def flow_fields_from_physical(self, d: dict, time: float):
        """ReadHDF5 (for/hdf5.f:296-544) from the dataset arrays of
        flow_fields_physical (P optional: without it POISSON_P_CHAN runs)."""
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        U, V, W = f(d["U"]), f(d["V"]), f(d["W"])
        TH = f(np.stack([d[f"TH{n + 1}"] for n in range(self.p.n_th)])) if self.p.n_th else None
        P = f(d["P"]) if "P" in d else None
        self._call("diablo_flow_fields_from_physical", _ptr(U), _ptr(V), _ptr(W),
                   None if TH is None else _ptr(TH), None if P is None else _ptr(P), time)

    def save_stats(self) -> dict:
        """SAVE_STATS_CHAN(FINAL=.FALSE.) + tkebudget_chan profiles
        (for/save_stats.f:4-690,963-1173): arrays over rows j = 0..NY+1 named
        as the reference's variables (scalar profiles as [N_TH][NY+2]), and
        the bulk values.  Applies the velocity BCs first and advances the
        running means, as the reference does."""
        L = self.p.ny + 2
        prof = np.zeros((len(_lib.PROFILES), L))
        prof_th = np.zeros((max(self.p.n_th, 1), len(_lib.PROFILES_TH), L))
        bulk = np.zeros(len(_lib.BULK))
        self._call("diablo_save_stats_chan", _ptr(prof), _ptr(prof_th), _ptr(bulk))
        out = {nm: prof[i] for i, nm in enumerate(_lib.PROFILES)}
        out.update({nm: prof_th[: self.p.n_th, i] for i, nm in enumerate(_lib.PROFILES_TH)})
        out.update({nm: float(v) for nm, v in zip(_lib.BULK, bulk)})
        return out

    def stats_means(self) -> dict:
        """NSAMPLES and the running means UBAR, VBAR, WBAR, THBAR that
        SAVE_STATS_CHAN(FINAL=.TRUE.) writes (rows 0..NY+1)."""
        L = self.p.ny + 2
        u, v, w = np.zeros(L), np.zeros(L), np.zeros(L)
        th = np.zeros((max(self.p.n_th, 1), L))
        n = ctypes.c_int()
        self._call("diablo_stats_means", _ptr(u), _ptr(v), _ptr(w), _ptr(th), ctypes.byref(n))
        return {"nsamples": n.value, "ubar": u, "vbar": v, "wbar": w, "thbar": th[: self.p.n_th]}

    def __init__(self, p: Params, gy, stream=None):
        if p.num_per_dir != 2:
            raise ValueError("Channel needs num_per_dir = 2")
        super().__init__(p, gy, stream)
        self.GY, self.GYF, self.DY, self.DYF = grid_metrics(gy)

    # ---- the reference's subroutines
    def rk_chan_1(self, time_step: int, rk_step: int):
        self._call("diablo_rk_chan_1", time_step, rk_step)

    def nu_t(self) -> np.ndarray:
        """NU_T of the last LES substep (physical, GY points)."""
        out = np.zeros(self.phys_shape)
        self._call("diablo_les_nu_t", _ptr(out), _lib.DG_HOST)
        return out

    def les_stats_request(self):
        """Record les_chan's plane means in the next LES substep."""
        self._call("diablo_les_stats_request")

    def les_stats(self) -> dict:
        """NU_T_MEAN ('nu_sgs') and EPS_SGS1_MEAN ('eps_sgs1'), rows 0..NY+1."""
        a, b = np.zeros(self.p.ny + 2), np.zeros(self.p.ny + 2)
        self._call("diablo_les_stats", _ptr(a), _ptr(b))
        return {"nu_sgs": a, "eps_sgs1": b}

    def les_tke(self) -> np.ndarray:
        """tkebudget_chan_les: epsilon_sgs, rows 1..NY (applies APPLY_BC_VEL)."""
        out = np.zeros(self.p.ny + 2)
        self._call("diablo_les_tke", _ptr(out))
        return out

    def rem_div_chan(self):
        self._call("diablo_rem_div_chan")

    def poisson_p_chan(self):
        self._call("diablo_poisson_p_chan")

    def apply_bc_vel(self):
        self._call("diablo_apply_bc_vel")

    def courant(self):
        self._call("diablo_courant")

    def step(self, time_step: int):
        for rk in (1, 2, 3):
            self.rk_chan_1(time_step, rk)
        self.advance_time()

    # ---- transforms on reference-layout host arrays
    def _ref_phys(self, v):
        shp = (self.p.ny + 2, self.p.nz + 2, self.p.nx + 2)
        return np.ascontiguousarray(v, dtype=np.float64).reshape(shp)

    def fft_xz_to_fourier(self, V: np.ndarray, VV: np.ndarray | None = None, jmin=0, jmax=None):
        """FFT_XZ_TO_FOURIER(V, VV, JMIN, JMAX) on reference-layout host arrays.
        V: (NY+2, NZ+2, NX+2) float64; returns VV (NY+2, NZ+2, NX/2+1) complex128."""
        jmax = self.p.ny + 1 if jmax is None else jmax
        V = self._ref_phys(V)
        if VV is None:
            VV = np.zeros((self.p.ny + 2, self.p.nz + 2, self.p.nx // 2 + 1), dtype=np.complex128)
        self._call("diablo_fft_xz_to_fourier", _ptr(V), _ptr(VV), jmin, jmax, _lib.DG_HOST)
        return VV

    def fft_xz_to_physical(self, VV: np.ndarray, V: np.ndarray | None = None, jmin=0, jmax=None):
        jmax = self.p.ny + 1 if jmax is None else jmax
        VV = np.ascontiguousarray(VV, dtype=np.complex128)
        if V is None:
            V = np.zeros((self.p.ny + 2, self.p.nz + 2, self.p.nx + 2), dtype=np.float64)
        self._call("diablo_fft_xz_to_physical", _ptr(VV), _ptr(V), jmin, jmax, _lib.DG_HOST)
        return V

    # ---- initial condition (CREATE_FLOW_CHAN tail, for/set_ics.f:109-182)
    def create_flow(self, u1, u2, u3, th=None):
        """Physical fields [NY+2][NZ][NX] -> spectral state: FFT, APPLY_BC_VEL,
        REM_DIV_CHAN, APPLY_BC_VEL (the SAVE_STATS_CHAN side effect)."""
        names = [("CU1", u1), ("CU2", u2), ("CU3", u3)]
        if th is not None:
            names += [(f"CTH{n}", th[n]) for n in range(self.p.n_th)]
        zero = np.zeros(self.spec_shape, dtype=np.complex128)
        for nm in ["CP", "CF1", "CF2", "CF3"] + [f"CFTH{n}" for n in range(self.p.n_th)]:
            self.set_field(nm, zero)
        for nm, a in names:
            self.set_field(nm, self.to_fourier(a))
        self.apply_bc_vel()
        self.rem_div_chan()
        self.apply_bc_vel()

    def to_fourier(self, phys: np.ndarray) -> np.ndarray:
        """Compact physical [NY+2][NZ][NX] -> compact spectral, via FFT_XZ_TO_FOURIER."""
        p = self.p
        V = np.zeros((p.ny + 2, p.nz + 2, p.nx + 2))
        V[:, : p.nz, : p.nx] = phys
        VV = self.fft_xz_to_fourier(V)
        return np.ascontiguousarray(VV[:, : p.tnkz + 1, : p.nkx + 1])

    def to_physical(self, spec: np.ndarray) -> np.ndarray:
        p = self.p
        VV = np.zeros((p.ny + 2, p.nz + 2, p.nx // 2 + 1), dtype=np.complex128)
        VV[:, : p.tnkz + 1, : p.nkx + 1] = spec
        V = self.fft_xz_to_physical(VV)
        return np.ascontiguousarray(V[:, : p.nz, : p.nx])


class Periodic(_Solver):
    """Device-resident triply periodic state driven through RK_PER_1."""

    def __init__(self, p: Params, stream=None):
        if p.num_per_dir != 3:
            raise ValueError("Periodic needs num_per_dir = 3")
        super().__init__(p, None, stream)

    def rk_per_1(self, rk_step: int):
        self._call("diablo_rk_per_1", rk_step)

    def rem_div_per(self):
        self._call("diablo_rem_div_per")

    def poisson_p_per(self):
        self._call("diablo_poisson_p_per")

    def step(self, time_step: int = 0):
        for rk in (1, 2, 3):
            self.rk_per_1(rk)
        self.advance_time()

    # ---- transforms
    def fft_xzy_to_fourier(self, U: np.ndarray, CU: np.ndarray | None = None):
        """FFT_XZY_TO_FOURIER(U, CU) on reference-layout host arrays.
        U: (NY+2, NZ+2, NX+2) float64; returns CU (NY+2, NZ+2, NX/2+1) complex128."""
        p = self.p
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(p.ny + 2, p.nz + 2, p.nx + 2)
        if CU is None:
            CU = np.zeros((p.ny + 2, p.nz + 2, p.nx // 2 + 1), dtype=np.complex128)
        self._call("diablo_fft_xzy_to_fourier", _ptr(U), _ptr(CU), _lib.DG_HOST)
        return CU

    def fft_xzy_to_physical(self, CU: np.ndarray, U: np.ndarray | None = None):
        p = self.p
        CU = np.ascontiguousarray(CU, dtype=np.complex128)
        if U is None:
            U = np.zeros((p.ny + 2, p.nz + 2, p.nx + 2), dtype=np.float64)
        self._call("diablo_fft_xzy_to_physical", _ptr(CU), _ptr(U), _lib.DG_HOST)
        return U

    def to_fourier(self, phys: np.ndarray) -> np.ndarray:
        """Physical [NY][NZ][NX] -> retained modes [TNKY+1][TNKZ+1][NKX+1]."""
        p = self.p
        U = np.zeros((p.ny + 2, p.nz + 2, p.nx + 2))
        U[: p.ny, : p.nz, : p.nx] = phys
        CU = self.fft_xzy_to_fourier(U)
        return np.ascontiguousarray(CU[: p.tnky + 1, : p.tnkz + 1, : p.nkx + 1])

    def to_physical(self, spec: np.ndarray) -> np.ndarray:
        p = self.p
        CU = np.zeros((p.ny + 2, p.nz + 2, p.nx // 2 + 1), dtype=np.complex128)
        CU[: p.tnky + 1, : p.tnkz + 1, : p.nkx + 1] = spec
        U = self.fft_xzy_to_physical(CU)
        return np.ascontiguousarray(U[: p.ny, : p.nz, : p.nx])

    def create_flow(self, u1, u2, u3, th=None):
        """CREATE_FLOW_PER tail (for/set_ics.f:278-319 then for/periodic.f
        REM_DIV_PER and POISSON_P_PER): physical [NY][NZ][NX] fields -> state."""
        zero = np.zeros(self.spec_shape, dtype=np.complex128)
        for nm in ["CP", "CF1", "CF2", "CF3"] + [f"CFTH{n}" for n in range(self.p.n_th)]:
            self.set_field(nm, zero)
        for nm, a in (("CU1", u1), ("CU2", u2), ("CU3", u3)):
            self.set_field(nm, self.to_fourier(a))
        if th is not None:
            for n in range(self.p.n_th):
                self.set_field(f"CTH{n}", self.to_fourier(th[n]))
        self.rem_div_per()
        self.poisson_p_per()


def thomas_real(a, b, c, g, ny: int, nx: int):
    """THOMAS_REAL(A,B,C,G,NY,NX) on host arrays shaped (NY+1, NX+1); returns
    (A, B, G) as modified by the reference routine."""
    L = _lib.load()
    arrs = [np.ascontiguousarray(x, dtype=np.float64).copy() for x in (a, b, c, g)]
    _lib.check("diablo_thomas_real",
               L.diablo_thomas_real(*[_ptr(x) for x in arrs], ny, nx, _lib.DG_HOST))
    return arrs[0], arrs[1], arrs[3]


def thomas_complex(a, b, c, g, ny: int, nx: int):
    L = _lib.load()
    arrs = [np.ascontiguousarray(x, dtype=np.float64).copy() for x in (a, b, c)]
    gg = np.ascontiguousarray(g, dtype=np.complex128).copy()
    _lib.check("diablo_thomas_complex",
               L.diablo_thomas_complex(*[_ptr(x) for x in arrs], _ptr(gg), ny, nx, _lib.DG_HOST))
    return arrs[0], arrs[1], gg
