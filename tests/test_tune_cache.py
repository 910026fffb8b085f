"""The autotuner's per-shape tuning cache: JSON load / save / lookup through
the C-ABI (no GPU needed: the table is host memory)."""
import json

import pytest

from diablo_b200 import _lib, configs


def test_cache_round_trip(tmp_path):
    p, _ = configs.kh_shear_layer(nx=64, ny=33, nz=16)
    key = f"{p.nx}x{p.ny}x{p.nz}_th{p.n_th}_fp64"
    src = tmp_path / "in.json"
    src.write_text(json.dumps({key: {"col_mt": 16, "xrow_chunk": 8, "ychunk": 0, "cn_mt": 2,
                                     "pdl": 1, "fft_plan": 1, "unknown_knob": 5}}))
    _lib.tune_cache_load(str(src))
    assert _lib.tune_cache_get(p, 0) == 16         # DG_TUNE_COL_MT
    assert _lib.tune_cache_get(p, 3) == 2          # DG_TUNE_CN_MT
    assert _lib.tune_cache_get(p, 6) == 1          # DG_TUNE_FFT_PLAN
    assert _lib.tune_cache_get(p.replace(precision=1), 0) is None
    out = tmp_path / "out.json"
    _lib.tune_cache_save(str(out))
    table = json.loads(out.read_text())
    assert table[key] == {"col_mt": 16, "xrow_chunk": 8, "ychunk": 0, "cn_mt": 2, "pdl": 1,
                          "fft_plan": 1}


def test_cache_rejects_malformed_file(tmp_path):
    p, _ = configs.kh_shear_layer(nx=32, ny=17, nz=16)
    key = f"{p.nx}x{p.ny}x{p.nz}_th{p.n_th}_fp64"
    good = tmp_path / "good.json"
    good.write_text(json.dumps({key: {"cn_mt": 8}}))
    _lib.tune_cache_load(str(good))
    assert _lib.tune_cache_get(p, 3) == 8
    bad = tmp_path / "bad.json"
    bad.write_text('{"' + key + '": {"cn_mt": "eight"}}')
    with pytest.raises(_lib.DiabloError):
        _lib.tune_cache_load(str(bad))
    assert _lib.tune_cache_get(p, 3) == 8          # the table is as it was
