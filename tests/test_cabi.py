"""The C-ABI library loads and exports every symbol include/diablo_b200.h
declares; without a GPU it refuses cleanly instead of crashing."""
import ctypes

import pytest

from diablo_b200 import _lib, configs
from diablo_b200.params import DgParams


def test_header_symbols_exported():
    L = _lib.load()
    names = _lib.declared_symbols()
    assert "diablo_rk_chan_1" in names and "diablo_fft_xz_to_fourier" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_params_struct_layout_matches_header():
    # the ctypes mirrors against the structs as the library compiled them
    from diablo_b200._lib import DgStats
    L = _lib.load()
    L.dg_abi_layout.restype = ctypes.c_int
    L.dg_abi_layout.argtypes = [ctypes.c_void_p, ctypes.c_int]
    n = L.dg_abi_layout(None, 0)
    buf = (ctypes.c_int64 * n)()
    assert L.dg_abi_layout(buf, n) == n == 11
    sizes = list(buf)
    assert sizes[0] == ctypes.sizeof(DgParams)
    assert sizes[1] == ctypes.sizeof(DgStats)
    names = ["nx", "nu", "f_type", "ubulk0", "th_bc_ymin", "epsilon_target", "les",
             "les_model_type", "create_new_flow"]
    assert sizes[2:] == [getattr(DgParams, f).offset for f in names]


def test_init_refuses_without_device_or_bad_args():
    L = _lib.load()
    p, gy = configs.kh_shear_layer(nx=32, ny=17, nz=16)
    bad = p.replace(nx=28)  # 28 = 4*7: no radix-7 pass
    h = ctypes.c_void_p()
    code = L.diablo_gpu_init(ctypes.byref(bad.to_struct(DgParams)), None, None, ctypes.byref(h))
    assert code in (2,)  # DG_ERR_DIMS (also checked before any device call)
    code = L.diablo_gpu_init(ctypes.byref(p.replace(num_per_dir=5).to_struct(DgParams)), None,
                             None, ctypes.byref(h))
    assert code == 1
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        import numpy as np
        g = np.ascontiguousarray(gy)
        code = L.diablo_gpu_init(ctypes.byref(p.to_struct(DgParams)),
                                 g.ctypes.data_as(ctypes.c_void_p), None, ctypes.byref(h))
        assert code == 7  # DG_ERR_NODEV
        assert b"device" in L.dg_last_error()


def test_mixed_precision_refuses_unsupported_sizes():
    L = _lib.load()
    import numpy as np
    p, gy = configs.kh_shear_layer(nx=36, ny=17, nz=18)
    g = np.ascontiguousarray(gy)
    h = ctypes.c_void_p()
    code = L.diablo_gpu_init(ctypes.byref(p.replace(precision=1).to_struct(DgParams)),
                             g.ctypes.data_as(ctypes.c_void_p), None, ctypes.byref(h))
    assert code == 2  # DG_ERR_DIMS, before any device call
    assert b"mixed precision" in L.dg_last_error()
    q, _ = configs.periodic_256(n=36)       # no FP32 product kernel for NX = 36
    code = L.diablo_gpu_init(ctypes.byref(q.replace(precision=1).to_struct(DgParams)), None, None,
                             ctypes.byref(h))
    assert code == 2
    code = L.diablo_gpu_init(ctypes.byref(q.replace(precision=2).to_struct(DgParams)), None, None,
                             ctypes.byref(h))
    assert code == 1


def test_state_bytes_estimate():
    from diablo_b200.serve import state_bytes
    p, _ = configs.channel_re180()
    b = state_bytes(p)
    m = 43 * 85 * 131 * 16                     # one retained-mode FP64 field
    assert 12 * m < b < 60 * m                  # state, work arrays, H and G planes
    assert state_bytes(p.replace(nx=64)) < b
