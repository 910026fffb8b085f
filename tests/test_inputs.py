"""Input parsers and grid tools against the reference's own fixtures
(tests/golden, generated by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from diablo_b200 import grid, params

GOLD = os.path.join(os.path.dirname(__file__), "golden")
KH = os.path.join(GOLD, "kh_input")


def test_grid_def_parsers():
    p = params.read_grid_def(os.path.join(KH, "grid_def.all"))
    assert (p.nx, p.ny, p.nz, p.n_th) == (128, 65, 16, 1)
    q = params.read_grid_def(os.path.join(KH, "grid_def"))
    assert (q.nx, q.ny, q.nz, q.n_th) == (128, 33, 16, 1)


def test_input_dat_and_input_chan():
    p = params.read_grid_def(os.path.join(KH, "grid_def.all"))
    p = params.read_input_dat(os.path.join(KH, "input.dat"), p, p.n_th)
    assert (p.nu, p.beta, p.lx, p.ly, p.lz) == (0.001, 1.0, 30.0, 20.0, 4.0)
    assert p.nu_v_scale == 1.0 and p.num_per_dir == 2
    assert p.delta_t == 0.1 and p.variable_dt == 1 and p.cfl == 0.5 and p.update_dt == 1
    assert p.ri[0] == 0.15 and p.pr[0] == 1.0
    assert p.les == 1 and p.create_new_flow == 1   # USE_LES, CREATE_NEW_FLOW
    p = params.read_input_chan(os.path.join(KH, "input_chan.dat"), p)
    assert p.les_model_type == 1
    assert (p.i_ro, p.grav_x, p.grav_y, p.grav_z) == (0.0, 0.0, 1.0, 0.0)
    assert (p.f_type, p.ubulk0, p.px0, p.omega0, p.amp_omega0) == (3, 0.0, -1.0, 6.28, 0.0)
    assert (p.u_bc_ymin, p.v_bc_ymin, p.w_bc_ymin) == (1, 0, 1)
    assert (p.u_bc_ymax, p.v_bc_ymax, p.w_bc_ymax) == (1, 0, 1)
    assert p.th_bc_ymin[0] == 1 and p.th_bc_ymax[0] == 1
    assert p.drhodx[0] == 0.0 and p.drhodz[0] == 0.0


def test_input_per_version_check():
    # the shipped KH_test/input_per.dat still says VERSION 1.0; the reference
    # STOPs on it ("Wrong input data format", for/periodic.f:443-444)
    p = params.Params(n_th=1)
    with pytest.raises(ValueError):
        params.read_input_per(os.path.join(KH, "input_per.dat"), p)


def test_create_grid_reproduces_kh_fixture():
    vals = np.loadtxt(os.path.join(GOLD, "kh_grid_y.txt"))
    g = grid.create_grid(2, 65, 20.0, 1.5)
    assert g.shape == vals.shape
    np.testing.assert_allclose(g, vals, rtol=0, atol=1e-13)


def test_grid_metrics_and_text_grid(tmp_path):
    gy = grid.create_grid(1, 33, 2.0, 1.75)
    GY, GYF, DY, DYF = grid.grid_metrics(gy)
    n = 33
    assert abs(GYF[1] + 1) < 1e-14 and abs(GYF[n] - 1) < 1e-14
    np.testing.assert_allclose(DY[1:], GYF[1:] - GYF[:-1])
    np.testing.assert_allclose(DYF[1: n + 1], GY[2:] - GY[1:-1])
    assert DYF[n + 1] == DYF[n]
    f = tmp_path / "ygrid.txt"
    grid.write_ygrid_txt(str(f), gy)
    np.testing.assert_allclose(grid.read_ygrid_txt(str(f), 33), gy, rtol=0, atol=0)
    with pytest.raises(ValueError):
        grid.read_ygrid_txt(str(f), 34)
