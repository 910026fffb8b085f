"""Named workloads (the benchmark configurations) as Params + grids.

kh_shear_layer   : NX=128, NZ=32, NY=65 uniform on [-10,10], Lx=4pi/0.44, Lz=Lx/4,
                   nu=1e-3, Pr=1, Ri=0.1, free-slip U/W, V=0, Dirichlet TH, dt=0.01.
channel_re180    : 128x129x128, Lx=4pi, Ly=2 (tanh stretch 1.75), Lz=4pi/3,
                   nu=1/180, constant pressure gradient PX0=-1, no-slip, CFL=0.5.
periodic_256     : 256^3 on [0,2pi]^3, nu=1e-3, decaying.
channel_re550    : 512x257x384, Lx=2pi, Ly=2 (tanh stretch 2.0), Lz=pi, one passive
                   scalar (Pr=0.71, Ri=0).
kh_les           : the reference's KH_test run (KH_test/input.dat, input_chan.dat,
                   grid_def.all, grid.h5): 128x65x16 stretched on [-10,10], Lx=30, Lz=4,
                   nu=1e-3, Ri=0.15, Pr=1, free-slip U/W, V=0, Neumann TH, CFL=0.5,
                   constant Smagorinsky LES.
"""
from __future__ import annotations

import math

from .grid import create_grid, uniform_grid
from .params import Params


def kh_shear_layer(nx=128, ny=65, nz=32):
    lx = 4 * math.pi / 0.44
    p = Params(nx=nx, ny=ny, nz=nz, n_th=1, num_per_dir=2, nu=1e-3, beta=1.0, lx=lx, ly=20.0,
               lz=lx / 4, delta_t=0.01, variable_dt=0, cfl=0.5, grav_y=1.0, f_type=0,
               u_bc_ymin=1, v_bc_ymin=0, w_bc_ymin=1, u_bc_ymax=1, v_bc_ymax=0, w_bc_ymax=1)
    p.ri[0] = 0.1
    p.pr[0] = 1.0
    p.th_bc_ymin[0] = 0
    p.th_bc_ymax[0] = 0
    p.th_bc_ymin_c1[0] = -1.0
    p.th_bc_ymax_c1[0] = 1.0
    return p, uniform_grid(ny, -10.0, 10.0)


def channel_re180(nx=128, ny=129, nz=128, cfl=0.5):
    p = Params(nx=nx, ny=ny, nz=nz, n_th=0, num_per_dir=2, nu=1.0 / 180.0, beta=1.0,
               lx=4 * math.pi, ly=2.0, lz=4 * math.pi / 3, delta_t=1e-3, variable_dt=1,
               update_dt=1, cfl=cfl, grav_y=1.0, f_type=1, ubulk0=15.6, px0=-1.0,
               u_bc_ymin=0, v_bc_ymin=0, w_bc_ymin=0, u_bc_ymax=0, v_bc_ymax=0, w_bc_ymax=0)
    return p, create_grid(1, ny, 2.0, 1.75)


def channel_re550(nx=512, ny=257, nz=384, cfl=0.5):
    p = Params(nx=nx, ny=ny, nz=nz, n_th=1, num_per_dir=2, nu=1.0 / 550.0, beta=1.0,
               lx=2 * math.pi, ly=2.0, lz=math.pi, delta_t=1e-3, variable_dt=1, update_dt=1,
               cfl=cfl, grav_y=1.0, f_type=1, ubulk0=18.3, px0=-1.0,
               u_bc_ymin=0, v_bc_ymin=0, w_bc_ymin=0, u_bc_ymax=0, v_bc_ymax=0, w_bc_ymax=0)
    p.pr[0] = 0.71
    p.ri[0] = 0.0
    p.th_bc_ymin[0] = 0
    p.th_bc_ymax[0] = 0
    p.th_bc_ymin_c1[0] = -1.0
    p.th_bc_ymax_c1[0] = 1.0
    return p, create_grid(1, ny, 2.0, 2.0)


def kh_les(nx=128, ny=65, nz=16):
    """The KH_test run with the subgrid model on from the first step (as after
    a restart; a new flow would wait 100 steps) on its stretched grid
    (KH_test/grid.h5: CREATE_GRID type 2, CS = 1.5)."""
    p = Params(nx=nx, ny=ny, nz=nz, n_th=1, num_per_dir=2, nu=1e-3, beta=1.0, lx=30.0, ly=20.0,
               lz=4.0, delta_t=0.1, variable_dt=1, update_dt=1, cfl=0.5, grav_y=1.0, f_type=0,
               u_bc_ymin=1, v_bc_ymin=0, w_bc_ymin=1, u_bc_ymax=1, v_bc_ymax=0, w_bc_ymax=1,
               les=1, les_model_type=1)
    p.ri[0] = 0.15
    p.pr[0] = 1.0
    p.th_bc_ymin[0] = 1
    p.th_bc_ymax[0] = 1
    return p, create_grid(2, ny, 20.0, 1.5)


def periodic_256(n=256, nu=1e-3, dt=2e-3):
    p = Params(nx=n, ny=n, nz=n, n_th=0, num_per_dir=3, nu=nu, beta=1.0, lx=2 * math.pi,
               ly=2 * math.pi, lz=2 * math.pi, delta_t=dt, variable_dt=0)
    return p, None
