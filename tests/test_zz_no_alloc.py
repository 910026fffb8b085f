"""The allocation-free FFT_XZ_TO_FOURIER entry point against the
handle-based one and the CPU oracle, through the C-ABI (needs a B200).

Collected last on purpose: it shares one fixed device array across calls,
and the two calls below run back to back on it with different sizes.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from diablo_b200 import _lib
from diablo_b200.grid import uniform_grid
from diablo_b200.params import Params

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_noalloc_matches_handle_entry_point_two_calls():
    import torch
    from diablo_b200.solver import Channel
    L = _lib.load()
    # call 1: 32 planes of 512 x 384, more than one chunk of the scratch, out
    # of place; call 2: 48 x 96, planes 1..9 of 11, in place (V and VV alias)
    cases = [((512, 384, 30), 0, 31, False), ((48, 96, 9), 1, 9, True)]
    stream = torch.cuda.current_stream()
    for (nx, nz, ny), jmin, jmax, inplace in cases:
        p = Params(nx=nx, ny=ny, nz=nz, lx=1.0, lz=1.0)
        ch = Channel(p, uniform_grid(ny, -1.0, 1.0))
        rng = np.random.default_rng(nx + nz + ny)
        V = np.zeros((ny + 2, nz + 2, nx + 2))
        V[:, :nz, :nx] = rng.standard_normal((ny + 2, nz, nx))
        want = ch.fft_xz_to_fourier(V, jmin=jmin, jmax=jmax)      # handle-based, host arrays
        ch.close()
        dV = torch.from_numpy(V).cuda()
        if inplace:
            dVV = dV
        else:
            dVV = torch.full((ny + 2, nz + 2, nx + 2), 7.0, dtype=torch.float64, device="cuda")
        code = L.diablo_fft_xz_to_fourier_noalloc(
            ctypes.c_void_p(dV.data_ptr()), ctypes.c_void_p(dVV.data_ptr()), nx, nz, ny, jmin, jmax,
            ctypes.c_void_p(stream.cuda_stream))
        assert code == 0, L.dg_last_error()
        torch.cuda.synchronize()
        got = dVV.cpu().numpy().view(np.complex128)
        planes = slice(jmin, jmax + 1)
        assert rel(got[planes], want[planes]) < 1e-14
        # retained block nonzero, everything else in the written planes zero
        assert np.all(got[planes][:, p.tnkz + 1:] == 0) and np.all(got[planes][:, :, p.nkx + 1:] == 0)
        # planes outside JMIN..JMAX untouched
        if inplace:
            assert np.array_equal(got[0], V.view(np.complex128)[0])
            assert np.array_equal(got[ny + 1], V.view(np.complex128)[ny + 1])
        if nx * nz <= 48 * 96:
            # the small case also against the CPU oracle's FFT_XZ_TO_FOURIER:
            # the retained block of every written plane, and zeros elsewhere
            ref = O.Oracle(p, uniform_grid(ny, -1.0, 1.0))
            spec = ref.to_fourier(np.ascontiguousarray(V[:, :nz, :nx]))
            ref.close()
            blk = got[planes][:, : p.tnkz + 1, : p.nkx + 1]
            assert rel(blk, spec[planes]) < 1e-14
            full = np.zeros_like(got[planes])
            full[:, : p.tnkz + 1, : p.nkx + 1] = spec[planes]
            assert rel(got[planes], full) < 1e-14


def test_noalloc_rejects_planes_beyond_its_scratch():
    import torch
    L = _lib.load()
    # one 4096 x 4096 plane needs ~90 MB of scratch; the check runs before
    # anything is queued, so a small buffer is enough to show the refusal
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptr = ctypes.c_void_p(buf.data_ptr())
    code = L.diablo_fft_xz_to_fourier_noalloc(ptr, ptr, 4096, 4096, 8, 0, 9, None)
    assert code == 2  # DG_ERR_DIMS
    assert b"DG_NOALLOC_SCRATCH_BYTES" in L.dg_last_error()


def test_noalloc_rejects_host_memory():
    """A host pointer would fault inside the kernels; the call refuses it
    before anything is queued."""
    L = _lib.load()
    host = np.zeros((11, 18, 34))
    hp = ctypes.c_void_p(host.ctypes.data)
    code = L.diablo_fft_xz_to_fourier_noalloc(hp, hp, 32, 16, 9, 0, 10, None)
    assert code == 1  # DG_ERR_ARG
    assert b"device" in L.dg_last_error()
