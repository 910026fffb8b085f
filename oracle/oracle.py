"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() (as the
checker) and bench.py's CPU-baseline leg.  See oracle.h for what it restates
and how it is pinned.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from diablo_b200.params import MAX_TH, Params

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

c_d, c_i, c_l = ctypes.c_double, ctypes.c_int, ctypes.c_long
P = ctypes.c_void_p


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("nx", c_i), ("ny", c_i), ("nz", c_i), ("n_th", c_i), ("num_per_dir", c_i),
        ("nu", c_d), ("beta", c_d), ("lx", c_d), ("ly", c_d), ("lz", c_d), ("nu_v_scale", c_d),
        ("delta_t", c_d), ("cfl", c_d), ("variable_dt", c_i), ("update_dt", c_i),
        ("i_ro", c_d), ("grav_x", c_d), ("grav_y", c_d), ("grav_z", c_d),
        ("f_type", c_i),
        ("ubulk0", c_d), ("px0", c_d), ("omega0", c_d), ("amp_omega0", c_d),
        ("u_bc_ymin", c_i), ("v_bc_ymin", c_i), ("w_bc_ymin", c_i),
        ("u_bc_ymax", c_i), ("v_bc_ymax", c_i), ("w_bc_ymax", c_i),
        ("u_bc_ymin_c1", c_d), ("v_bc_ymin_c1", c_d), ("w_bc_ymin_c1", c_d),
        ("u_bc_ymax_c1", c_d), ("v_bc_ymax_c1", c_d), ("w_bc_ymax_c1", c_d),
        ("th_bc_ymin", c_i * MAX_TH), ("th_bc_ymax", c_i * MAX_TH),
        ("th_bc_ymin_c1", c_d * MAX_TH), ("th_bc_ymax_c1", c_d * MAX_TH),
        ("ri", c_d * MAX_TH), ("pr", c_d * MAX_TH), ("drhodx", c_d * MAX_TH),
        ("drhodz", c_d * MAX_TH), ("background_grad", c_i * MAX_TH),
        ("epsilon_target", c_d),
        ("les", c_i), ("les_model_type", c_i), ("create_new_flow", c_i),
    ]


class OrcStats(ctypes.Structure):
    _fields_ = [("ubulk", c_d), ("urms_b", c_d), ("vrms_b", c_d), ("wrms_b", c_d),
                ("ke", c_d), ("div_max", c_d), ("thrms_b", c_d * MAX_TH),
                ("th_var", c_d * MAX_TH)]


# profile rows of orc_save_stats_chan, in the order of ORC_PR_* / ORC_PRT_*
PROFILES = ("ume", "vme", "wme", "urms", "vrms", "wrms", "uv", "uw", "wv", "dudy", "dwdy", "cp",
            "shear", "omega_x", "omega_y", "omega_z", "epsilon")
PROFILES_TH = ("thme", "dthdy", "thrms", "thv", "pe_diss")


def build(quiet: bool = True) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    r = subprocess.run(["make", "-s", "-C", _HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), P]
        L.orc_destroy.argtypes = [P]
        for f in ("orc_nkx", "orc_tnkz", "orc_tnky"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = c_i
        for f in ("orc_spec_size", "orc_phys_size"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = c_l
        L.orc_get_field.argtypes = [P, c_i, P]
        L.orc_set_field.argtypes = [P, c_i, P]
        L.orc_get_grid.argtypes = [P, P, P, P, P]
        L.orc_set_time.argtypes = [P, c_d, c_d]
        L.orc_get_time.argtypes = [P, P, P]
        L.orc_fft_xz_to_fourier.argtypes = [P, P, P, c_i, c_i]
        L.orc_fft_xz_to_physical.argtypes = [P, P, P, c_i, c_i]
        L.orc_fft_xzy_to_fourier.argtypes = [P, P, P]
        L.orc_fft_xzy_to_physical.argtypes = [P, P, P]
        L.orc_fft1d.argtypes = [c_i, P, c_i]
        L.orc_thomas_real.argtypes = [P, P, P, P, c_i, c_i]
        L.orc_thomas_complex.argtypes = [P, P, P, P, c_i, c_i]
        L.orc_rk_chan_1.argtypes = [P, c_i, c_i]
        for f in ("orc_rem_div_chan", "orc_poisson_p_chan", "orc_apply_bc_vel", "orc_courant",
                  "orc_rem_div_per", "orc_poisson_p_per"):
            getattr(L, f).argtypes = [P]
        L.orc_create_flow_chan.argtypes = [P, P, P, P, P]
        L.orc_create_flow_per.argtypes = [P, P, P, P]
        L.orc_rk_per_1.argtypes = [P, c_i]
        L.orc_stats_chan.argtypes = [P, ctypes.POINTER(OrcStats)]
        L.orc_stats_per.argtypes = [P, ctypes.POINTER(OrcStats)]
        L.orc_div_max_chan.argtypes = [P]
        L.orc_div_max_chan.restype = c_d
        L.orc_div_max_per.argtypes = [P]
        L.orc_div_max_per.restype = c_d
        L.orc_save_stats_chan.argtypes = [P, P, P, P]
        L.orc_stats_means_update.argtypes = [P, c_i, P, P, P, P]
        L.orc_set_threads.argtypes = [c_i]
        L.orc_get_nu_t.argtypes = [P, P]
        L.orc_les_stats_request.argtypes = [P]
        L.orc_les_stats.argtypes = [P, P, P]
        L.orc_tkebudget_chan_les.argtypes = [P, P]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(P)


FIELD = {"CU1": 0, "CU2": 1, "CU3": 2, "CP": 3, "CF1": 4, "CF2": 5, "CF3": 6, "CR1": 7}


def field_id(name: str) -> int:
    if name.startswith("CTH"):
        return 16 + int(name[3:] or 0)
    if name.startswith("CFTH"):
        return 32 + int(name[4:] or 0)
    return FIELD[name]


class Oracle:
    """One oracle instance (channel or periodic)."""

    def __init__(self, p: Params, gy: np.ndarray | None = None, threads: int = 0):
        self.p = p
        L = lib()
        if threads:
            L.orc_set_threads(threads)
        self._op = p.to_struct(OrcParams)
        gyp = None
        if gy is not None:
            self._gy = np.ascontiguousarray(gy, dtype=np.float64)
            gyp = _ptr(self._gy)
        self.h = L.orc_create(ctypes.byref(self._op), gyp)
        if not self.h:
            raise ValueError("ERROR: LES_MODEL_TYPE=2, 3 not supported yet in MPI")
        self.spec_shape = p.spec_shape()
        self.phys_shape = p.phys_shape()

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- fields
    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.spec_shape, dtype=np.complex128)
        if lib().orc_get_field(self.h, field_id(name), _ptr(out)) != 0:
            raise KeyError(name)
        return out

    def set(self, name: str, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.complex128).reshape(self.spec_shape)
        if lib().orc_set_field(self.h, field_id(name), _ptr(a)) != 0:
            raise KeyError(name)

    def state(self):
        names = ["CU1", "CU2", "CU3", "CP", "CF1", "CF2", "CF3"]
        names += [f"CTH{n}" for n in range(self.p.n_th)]
        names += [f"CFTH{n}" for n in range(self.p.n_th)]
        return {n: self.get(n) for n in names}

    def nu_t(self) -> np.ndarray:
        """NU_T (physical, GY points) after the last LES substep."""
        out = np.zeros(self.phys_shape)
        if lib().orc_get_nu_t(self.h, _ptr(out)) != 0:
            raise ValueError("no LES state")
        return out

    def les_stats_request(self):
        lib().orc_les_stats_request(self.h)

    def les_stats(self) -> dict:
        """NU_T_MEAN, EPS_SGS1_MEAN (rows 0..NY+1) of the requested substep."""
        a, b = np.zeros(self.p.ny + 2), np.zeros(self.p.ny + 2)
        if lib().orc_les_stats(self.h, _ptr(a), _ptr(b)) != 0:
            raise ValueError("no LES statistics recorded")
        return {"nu_sgs": a, "eps_sgs1": b}

    def tkebudget_chan_les(self) -> np.ndarray:
        """epsilon_sgs (rows 1..NY; sums over each plane) after APPLY_BC_VEL."""
        out = np.zeros(self.p.ny + 2)
        lib().orc_tkebudget_chan_les(self.h, _ptr(out))
        return out

    def set_state(self, st: dict):
        for k, v in st.items():
            self.set(k, v)

    def grid(self):
        n = self.p.ny + 2
        a = [np.zeros(n) for _ in range(4)]
        lib().orc_get_grid(self.h, *[_ptr(x) for x in a])
        return a

    def set_time(self, time: float, dt: float):
        lib().orc_set_time(self.h, time, dt)

    def get_time(self):
        t, d = c_d(), c_d()
        lib().orc_get_time(self.h, ctypes.byref(t), ctypes.byref(d))
        return t.value, d.value

    # --- transforms
    def to_fourier(self, phys: np.ndarray, jmin: int = 0, jmax: int | None = None) -> np.ndarray:
        ph = np.ascontiguousarray(phys, dtype=np.float64)
        if self.p.num_per_dir == 3:
            out = np.zeros(self.spec_shape, dtype=np.complex128)
            lib().orc_fft_xzy_to_fourier(self.h, _ptr(ph), _ptr(out))
            return out
        jmax = self.p.ny + 1 if jmax is None else jmax
        out = np.zeros(self.spec_shape, dtype=np.complex128)
        lib().orc_fft_xz_to_fourier(self.h, _ptr(ph), _ptr(out), jmin, jmax)
        return out

    def to_physical(self, spec: np.ndarray, jmin: int = 0, jmax: int | None = None) -> np.ndarray:
        sp = np.ascontiguousarray(spec, dtype=np.complex128)
        out = np.zeros(self.phys_shape, dtype=np.float64)
        if self.p.num_per_dir == 3:
            lib().orc_fft_xzy_to_physical(self.h, _ptr(sp), _ptr(out))
            return out
        jmax = self.p.ny + 1 if jmax is None else jmax
        lib().orc_fft_xz_to_physical(self.h, _ptr(sp), _ptr(out), jmin, jmax)
        return out

    # --- stepping
    def rk_chan_1(self, time_step: int, rk_step: int):
        lib().orc_rk_chan_1(self.h, time_step, rk_step)

    def rk_per_1(self, rk_step: int):
        lib().orc_rk_per_1(self.h, rk_step)

    def step(self, time_step: int):
        """One full RK3 step as the driver does (for/diablo.f:70-84,109)."""
        for rk in (1, 2, 3):
            if self.p.num_per_dir == 3:
                self.rk_per_1(rk)
            else:
                self.rk_chan_1(time_step, rk)
        t, dt = self.get_time()
        self.set_time(t + dt, dt)

    def rem_div_chan(self):
        lib().orc_rem_div_chan(self.h)

    def poisson_p_chan(self):
        lib().orc_poisson_p_chan(self.h)

    def apply_bc_vel(self):
        lib().orc_apply_bc_vel(self.h)

    def rem_div_per(self):
        lib().orc_rem_div_per(self.h)

    def poisson_p_per(self):
        lib().orc_poisson_p_per(self.h)

    def create_flow_chan(self, u1, u2, u3, th=None):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (u1, u2, u3)]
        t = None if th is None else np.ascontiguousarray(th, dtype=np.float64)
        lib().orc_create_flow_chan(self.h, *[_ptr(x) for x in a], None if t is None else _ptr(t))

    def create_flow_per(self, u1, u2, u3):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (u1, u2, u3)]
        lib().orc_create_flow_per(self.h, *[_ptr(x) for x in a])

    def stats(self) -> dict:
        s = OrcStats()
        if self.p.num_per_dir == 3:
            lib().orc_stats_per(self.h, ctypes.byref(s))
        else:
            lib().orc_stats_chan(self.h, ctypes.byref(s))
        d = {k: getattr(s, k) for k in ("ubulk", "urms_b", "vrms_b", "wrms_b", "ke", "div_max")}
        d["thrms_b"] = list(s.thrms_b)[: self.p.n_th]
        d["th_var"] = list(s.th_var)[: self.p.n_th]
        return d

    def save_stats_chan(self) -> dict:
        """SAVE_STATS_CHAN + tkebudget_chan profiles (see oracle.h); runs
        APPLY_BC_VEL on the state first, as the reference does."""
        L = self.p.ny + 2
        prof = np.zeros((len(PROFILES), L))
        prof_th = np.zeros((max(self.p.n_th, 1), len(PROFILES_TH), L))
        bulk = np.zeros(5)
        lib().orc_save_stats_chan(self.h, _ptr(prof), _ptr(prof_th), _ptr(bulk))
        out = {nm: prof[i] for i, nm in enumerate(PROFILES)}
        out.update({nm: prof_th[: self.p.n_th, i] for i, nm in enumerate(PROFILES_TH)})
        out.update(dict(zip(("ubulk", "uc", "urms_b", "vrms_b", "wrms_b"), bulk)))
        return out

    def stats_means_update(self, nsamples: int, ubar, vbar, wbar, thbar):
        """SAVE_STATS_CHAN's running means (in place; REAL*4 weights)."""
        lib().orc_stats_means_update(self.h, nsamples, _ptr(ubar), _ptr(vbar), _ptr(wbar),
                                     _ptr(thbar))

    def div_max(self) -> float:
        if self.p.num_per_dir == 3:
            return lib().orc_div_max_per(self.h)
        return lib().orc_div_max_chan(self.h)


def fft1d(x: np.ndarray, sign: int) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().orc_fft1d(a.size, _ptr(a), sign)
    return a


def thomas_real(a, b, c, g, ny, nx):
    arrs = [np.ascontiguousarray(x, dtype=np.float64).copy() for x in (a, b, c, g)]
    lib().orc_thomas_real(*[_ptr(x) for x in arrs], ny, nx)
    return arrs[3]


def thomas_complex(a, b, c, g, ny, nx):
    arrs = [np.ascontiguousarray(x, dtype=np.float64).copy() for x in (a, b, c)]
    gg = np.ascontiguousarray(g, dtype=np.complex128).copy()
    lib().orc_thomas_complex(*[_ptr(x) for x in arrs], _ptr(gg), ny, nx)
    return gg
