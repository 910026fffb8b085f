"""ctypes binding of libdiablo_b200.so (the C-ABI declared in include/diablo_b200.h).

The shared library is built in-tree by ``diablo_b200.build.build_library`` (or
``__graft_entry__.build()``).  There is no CPU fallback: if the library or a
B200 is missing, every solver call raises.
"""
from __future__ import annotations

import ctypes
import os
import re

from .params import MAX_TH, DgParams

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdiablo_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "diablo_b200.h")

DG_OK = 0
ERRORS = {1: "DG_ERR_ARG", 2: "DG_ERR_DIMS", 3: "DG_ERR_OOM", 4: "DG_ERR_CUDA", 5: "DG_ERR_NAN",
          6: "DG_ERR_TIMEOUT", 7: "DG_ERR_NODEV"}
DG_HOST, DG_DEVICE = 0, 1
DG_LAYOUT_COMPACT, DG_LAYOUT_REFERENCE, DG_LAYOUT_REFERENCE_RETAINED = 0, 1, 2
# rows of diablo_save_stats_chan's profiles (DG_PR_* and DG_PRT_* in the header)
PROFILES = ("ume", "vme", "wme", "urms", "vrms", "wrms", "uv", "uw", "wv", "dudy", "dwdy", "cp",
            "shear", "omega_x", "omega_y", "omega_z", "epsilon")
PROFILES_TH = ("thme", "dthdy", "thrms", "thv", "pe_diss")
BULK = ("ubulk", "uc", "urms_b", "vrms_b", "wrms_b")

FIELD_IDS = {"CU1": 0, "CU2": 1, "CU3": 2, "CP": 3, "CF1": 4, "CF2": 5, "CF3": 6, "CR1": 7}


def field_id(name: str) -> int:
    if name.startswith("CFTH"):
        return 32 + int(name[4:] or 0)
    if name.startswith("CTH"):
        return 16 + int(name[3:] or 0)
    return FIELD_IDS[name]


class DgStats(ctypes.Structure):
    _fields_ = [("ubulk", ctypes.c_double), ("urms_b", ctypes.c_double),
                ("vrms_b", ctypes.c_double), ("wrms_b", ctypes.c_double),
                ("ke", ctypes.c_double), ("div_max", ctypes.c_double),
                ("thrms_b", ctypes.c_double * MAX_TH), ("th_var", ctypes.c_double * MAX_TH)]


class DiabloError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed: {ERRORS.get(code, code)}: {msg}")
        self.code = code


def declared_symbols(header: str = HEADER_PATH):
    """Function names declared in the public header."""
    txt = open(header).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:diablo|dg)_[a-z0-9_]+)\s*\(", txt)))


_lib = None


def load(path: str = LIB_PATH):
    """Load the library (once) and declare argument types."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    L = ctypes.CDLL(path)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.dg_version.restype = I
    L.dg_last_error.restype = ctypes.c_char_p
    L.dg_kernel_launches.restype = ctypes.c_int64
    L.diablo_gpu_init.argtypes = [ctypes.POINTER(DgParams), P, P, ctypes.POINTER(P)]
    sigs = {
        "diablo_gpu_finalize": [P], "diablo_synchronize": [P],
        "diablo_set_time": [P, D, D],
        "diablo_get_time": [P, ctypes.POINTER(D), ctypes.POINTER(D)],
        "diablo_advance_time": [P],
        "diablo_set_field": [P, I, P, I, I], "diablo_get_field": [P, I, P, I, I],
        "diablo_set_fields": [P, I, P, P, I, I], "diablo_get_fields": [P, I, P, P, I, I],
        "diablo_rk_chan_1": [P, I, I], "diablo_les_nu_t": [P, P, I], "diablo_les_stats_request": [P],
        "diablo_les_stats": [P, P, P], "diablo_les_tke": [P, P], "diablo_rem_div_chan": [P], "diablo_poisson_p_chan": [P],
        "diablo_apply_bc_vel": [P], "diablo_courant": [P],
        "diablo_fft_xz_to_fourier": [P, P, P, I, I, I],
        "diablo_fft_xz_to_physical": [P, P, P, I, I, I],
        "diablo_thomas_real": [P, P, P, P, I, I, I],
        "diablo_thomas_complex": [P, P, P, P, I, I, I],
        "diablo_rk_per_1": [P, I], "diablo_rem_div_per": [P], "diablo_poisson_p_per": [P],
        "diablo_fft_xzy_to_fourier": [P, P, P, I], "diablo_fft_xzy_to_physical": [P, P, P, I],
        "diablo_fft_xz_to_fourier_noalloc": [P, P, I, I, I, I, I, P],
        "dg_timing_enable": [P, I], "diablo_step": [P, I, I],
        "dg_tune_set": [P, I, I], "dg_tune_get": [P, I, ctypes.POINTER(I)],
        "dg_autotune": [P, I], "dg_tune_lookup": [P, ctypes.POINTER(I)],
        "dg_tune_cache_get": [P, I, ctypes.POINTER(I)], "dg_tune_cache_save": [ctypes.c_char_p],
        "dg_tune_cache_load": [ctypes.c_char_p],
        "dg_server_create": [I, D, I, ctypes.POINTER(P)],
        "dg_server_submit": [P, P, P, P, I, I, ctypes.POINTER(ctypes.c_int64)],
        "dg_server_wait": [P, ctypes.c_int64, P, P],
        "dg_server_query": [P, P], "dg_server_destroy": [P], "dg_server_config": [P, I, I],
        "dg_timing_read": [P, I, ctypes.c_char_p, I, ctypes.POINTER(ctypes.c_int64),
                           ctypes.POINTER(D)],
        "diablo_stats": [P, ctypes.POINTER(DgStats)],
        "diablo_save_stats_chan": [P, P, P, P],
        "diablo_save_flow": [P, I, ctypes.c_char_p, P],
        "diablo_read_flow": [P, ctypes.c_char_p, P, ctypes.POINTER(I)],
        "diablo_flow_fields_physical": [P, P, P, P, P, P],
        "diablo_flow_fields_from_physical": [P, P, P, P, P, P, D],
        "diablo_stats_means": [P, P, P, P, P, ctypes.POINTER(I)],
    }
    L.dg_state_bytes.argtypes = [P]
    L.dg_state_bytes.restype = ctypes.c_int64
    for name, args in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = I
    _lib = L
    return L


def check(fn: str, code: int):
    if code != DG_OK:
        msg = load().dg_last_error().decode(errors="replace")
        raise DiabloError(fn, code, msg)


def kernel_launches() -> int:
    return int(load().dg_kernel_launches())


def tune_cache_save(path: str):
    """Write the process-wide tuning cache (dg_tune_cache_save) as JSON."""
    L = load()
    check("dg_tune_cache_save", L.dg_tune_cache_save(os.fsencode(path)))


def tune_cache_load(path: str):
    """Merge a JSON tuning cache into the process-wide one."""
    L = load()
    check("dg_tune_cache_load", L.dg_tune_cache_load(os.fsencode(path)))


def tune_cache_get(p, key: int):
    """One stored tunable for the shape of params p, or None."""
    L = load()
    v = ctypes.c_int()
    if L.dg_tune_cache_get(ctypes.byref(p.to_struct(DgParams)), key, ctypes.byref(v)) != 0:
        return None
    return v.value
