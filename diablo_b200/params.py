"""Run parameters and the reference's input-file parsers.

``Params`` carries what the reference keeps in COMMON /INPUT/, /SCALAR_VARS/,
/GEOPHYS_VARS/, /OSCILL_VARS/, /VARIABLE_VISC/ and /DRHODX_VARS/
(``for/header:83-186,289-302``) plus the compile-time grid (``grid_def``).
The parsers read the reference's fixed-line-count text files exactly as its
list-directed READs do: ``input.dat`` (``for/diablo_io.f:11-46``),
``input_chan.dat`` (``for/channel.f:1463-1509``), ``input_per.dat``
(``for/periodic.f:434-455``) and ``grid_def`` (``PARAMETER`` lines).
"""
from __future__ import annotations

import ctypes
import dataclasses
import re
from dataclasses import dataclass, field
from typing import List

MAX_TH = 4

__all__ = ["Params", "MAX_TH", "read_input_dat", "read_input_chan", "read_input_per",
           "read_grid_def", "DgParams"]


@dataclass
class Params:
    nx: int = 128
    ny: int = 65
    nz: int = 32
    n_th: int = 0
    num_per_dir: int = 2
    precision: int = 0              # 0 = plain FP64, 1 = mixed (FP32 FFT/products)
    nu: float = 1e-3
    beta: float = 1.0
    lx: float = 1.0
    ly: float = 2.0
    lz: float = 1.0
    nu_v_scale: float = 1.0
    delta_t: float = 1e-2
    cfl: float = 0.5
    variable_dt: int = 0
    update_dt: int = 1
    i_ro: float = 0.0
    grav_x: float = 0.0
    grav_y: float = 1.0
    grav_z: float = 0.0
    f_type: int = 0
    ubulk0: float = 0.0
    px0: float = 0.0
    omega0: float = 0.0
    amp_omega0: float = 0.0
    u_bc_ymin: int = 0
    v_bc_ymin: int = 0
    w_bc_ymin: int = 0
    u_bc_ymax: int = 0
    v_bc_ymax: int = 0
    w_bc_ymax: int = 0
    u_bc_ymin_c1: float = 0.0
    v_bc_ymin_c1: float = 0.0
    w_bc_ymin_c1: float = 0.0
    u_bc_ymax_c1: float = 0.0
    v_bc_ymax_c1: float = 0.0
    w_bc_ymax_c1: float = 0.0
    th_bc_ymin: List[int] = field(default_factory=lambda: [0] * MAX_TH)
    th_bc_ymax: List[int] = field(default_factory=lambda: [0] * MAX_TH)
    th_bc_ymin_c1: List[float] = field(default_factory=lambda: [0.0] * MAX_TH)
    th_bc_ymax_c1: List[float] = field(default_factory=lambda: [0.0] * MAX_TH)
    ri: List[float] = field(default_factory=lambda: [0.0] * MAX_TH)
    pr: List[float] = field(default_factory=lambda: [1.0] * MAX_TH)
    drhodx: List[float] = field(default_factory=lambda: [0.0] * MAX_TH)
    drhodz: List[float] = field(default_factory=lambda: [0.0] * MAX_TH)
    background_grad: List[int] = field(default_factory=lambda: [0] * MAX_TH)
    epsilon_target: float = 0.0
    les: int = 0                    # USE_LES (input.dat)
    les_model_type: int = 1         # input_chan.dat; the MPI build runs only 1
    create_new_flow: int = 0        # input.dat; the subgrid model waits 100 steps

    # derived sizes (for/header:22-28)
    @property
    def nkx(self) -> int:
        return self.nx // 3

    @property
    def nkz(self) -> int:
        return self.nz // 3

    @property
    def tnkz(self) -> int:
        return 2 * (self.nz // 3)

    @property
    def nky(self) -> int:
        return self.ny // 3

    @property
    def tnky(self) -> int:
        return 2 * (self.ny // 3)

    def spec_shape(self):
        """(planes, TNKZ+1, NKX+1) of one retained-mode spectral field."""
        if self.num_per_dir == 3:
            return (self.tnky + 1, self.tnkz + 1, self.nkx + 1)
        return (self.ny + 2, self.tnkz + 1, self.nkx + 1)

    def phys_shape(self):
        if self.num_per_dir == 3:
            return (self.ny, self.nz, self.nx)
        return (self.ny + 2, self.nz, self.nx)

    def replace(self, **kw) -> "Params":
        return dataclasses.replace(self, **kw)

    def to_struct(self, cls):
        """Fill a ctypes.Structure whose field names match ours."""
        s = cls()
        for name, _t in cls._fields_:
            if name.startswith("_pad"):
                continue
            v = getattr(self, name)
            if isinstance(v, list):
                arr = getattr(s, name)
                for i, x in enumerate(v[:len(arr)]):
                    arr[i] = x
            else:
                setattr(s, name, v)
        return s


def _c_fields():
    d, i = ctypes.c_double, ctypes.c_int32
    return [
        ("nx", i), ("ny", i), ("nz", i), ("n_th", i), ("num_per_dir", i), ("precision", i),
        ("nu", d), ("beta", d), ("lx", d), ("ly", d), ("lz", d), ("nu_v_scale", d),
        ("delta_t", d), ("cfl", d), ("variable_dt", i), ("update_dt", i),
        ("i_ro", d), ("grav_x", d), ("grav_y", d), ("grav_z", d),
        ("f_type", i), ("_pad0", i),
        ("ubulk0", d), ("px0", d), ("omega0", d), ("amp_omega0", d),
        ("u_bc_ymin", i), ("v_bc_ymin", i), ("w_bc_ymin", i),
        ("u_bc_ymax", i), ("v_bc_ymax", i), ("w_bc_ymax", i),
        ("u_bc_ymin_c1", d), ("v_bc_ymin_c1", d), ("w_bc_ymin_c1", d),
        ("u_bc_ymax_c1", d), ("v_bc_ymax_c1", d), ("w_bc_ymax_c1", d),
        ("th_bc_ymin", i * MAX_TH), ("th_bc_ymax", i * MAX_TH),
        ("th_bc_ymin_c1", d * MAX_TH), ("th_bc_ymax_c1", d * MAX_TH),
        ("ri", d * MAX_TH), ("pr", d * MAX_TH), ("drhodx", d * MAX_TH), ("drhodz", d * MAX_TH),
        ("background_grad", i * MAX_TH),
        ("epsilon_target", d),
        ("les", i), ("les_model_type", i), ("create_new_flow", i), ("_pad1", i),
    ]


class DgParams(ctypes.Structure):
    """Mirror of ``dg_params`` in include/diablo_b200.h."""
    _fields_ = _c_fields()


# ---------------------------------------------------------------- parsers
def _data_lines(path):
    with open(path) as f:
        return [ln.rstrip("\n") for ln in f]


def _tok(line):
    out = []
    for t in line.replace(",", " ").split():
        tl = t.strip().strip("'\"")
        out.append(tl)
    return out


def _f(t):
    return float(t.replace("D", "E").replace("d", "e"))


def _b(t):
    t = t.upper().strip(".")
    if t in ("TRUE", "T"):
        return True
    if t in ("FALSE", "F"):
        return False
    raise ValueError(f"not a Fortran logical: {t}")


def read_input_dat(path, p: Params | None = None, n_th: int | None = None) -> Params:
    """input.dat (for/diablo_io.f:18-46); N_TH comes from grid_def."""
    p = p or Params()
    if n_th is not None:
        p.n_th = n_th
    L = _data_lines(path)
    t = _tok(L[4])
    version = float(t[1])
    if version != 2.0:
        raise ValueError("Wrong input data format.")
    t = _tok(L[8])
    p.nu, p.beta, p.lx, p.ly, p.lz = map(_f, t[:5])
    p.nu_v_scale = _f(_tok(L[10])[0])
    p.les = int(_b(_tok(L[6])[1]))
    t = _tok(L[12])
    p.num_per_dir = int(t[0])
    p.create_new_flow = int(_b(t[1]))
    t = _tok(L[14])
    p.delta_t = _f(t[2])
    p.variable_dt = int(_b(t[4]))
    p.cfl = _f(t[5])
    p.update_dt = int(t[6])
    line = 18                          # first line of the 6-line block per scalar
    for n in range(p.n_th):
        ri_pr = _tok(L[line + 5])
        p.ri[n], p.pr[n] = _f(ri_pr[0]), _f(ri_pr[1])
        line += 6
    return p


def read_input_chan(path, p: Params) -> Params:
    """input_chan.dat (for/channel.f:1466-1509)."""
    L = _data_lines(path)
    if float(_tok(L[4])[0]) != 2.0:
        raise ValueError("Wrong input data format input_chan")
    p.les_model_type = int(_tok(L[8])[0])
    t = _tok(L[12])
    p.i_ro = _f(t[0])
    t = _tok(L[14])
    p.grav_x, p.grav_y, p.grav_z = map(_f, t[:3])
    t = _tok(L[16])
    p.f_type = int(t[0])
    p.ubulk0, p.px0, p.omega0, p.amp_omega0 = map(_f, t[1:5])
    rows = [("u", "ymin"), ("v", "ymin"), ("w", "ymin"), ("u", "ymax"), ("v", "ymax"),
            ("w", "ymax")]
    for r, (c, side) in enumerate(rows):
        t = _tok(L[18 + 2 * r])
        setattr(p, f"{c}_bc_{side}", int(t[0]))
        setattr(p, f"{c}_bc_{side}_c1", _f(t[1]))
    line = 30                          # first line of the 6-line block per scalar
    for n in range(p.n_th):
        t = _tok(L[line + 1])
        p.th_bc_ymin[n], p.th_bc_ymin_c1[n] = int(t[0]), _f(t[1])
        t = _tok(L[line + 3])
        p.th_bc_ymax[n], p.th_bc_ymax_c1[n] = int(t[0]), _f(t[1])
        t = _tok(L[line + 5])
        p.drhodx[n], p.drhodz[n] = _f(t[0]), _f(t[1])
        line += 6
    return p


def read_input_per(path, p: Params) -> Params:
    """input_per.dat (for/periodic.f:437-455)."""
    L = _data_lines(path)
    if float(_tok(L[4])[0]) != 2.0:
        raise ValueError("Wrong input data format input_per")
    line = 12                          # first line of the 2-line block per scalar
    for n in range(p.n_th):
        p.background_grad[n] = int(_b(_tok(L[line + 1])[0]))
        line += 2
    return p


def read_grid_def(path, p: Params | None = None) -> Params:
    """grid_def: ``PARAMETER (NX=128)`` lines for NX, NY, NZ, N_TH."""
    p = p or Params()
    txt = open(path).read()
    for name in ("NX", "NY", "NZ", "N_TH"):
        m = re.search(r"PARAMETER\s*\(\s*%s\s*=\s*(\d+)\s*\)" % name, txt, re.I)
        if m:
            setattr(p, name.lower(), int(m.group(1)))
    return p
