"""Flow files as the reference names and lays them out.

* Unformatted (for/diablo_io.f:201-404): ``Channel.save_flow`` /
  ``read_flow`` (also ``Periodic``) write and read them through the C-ABI;
  ``reference_names`` gives the reference's file names.
* HDF5 (for/hdf5.f:5-544): ``write_h5`` / ``read_h5`` put the arrays of
  ``Channel.flow_fields_physical`` into the reference's layout (group
  ``Timestep`` with attribute ``Time``, datasets U, V, W, TH1.., P; file
  attribute ``Resolution``).  They need h5py, which this image lacks; the
  arrays themselves come from the library either way.
"""
from __future__ import annotations

import time as _time


def reference_names(final: bool, n_th: int):
    """(velocity file, [scalar files]) of SAVE_FLOW (for/diablo_io.f:341-366)."""
    ext = "res" if final else "saved"
    return f"diablo.{ext}", [f"diablo_th{n + 1:02d}.{ext}" for n in range(n_th)]


def start_names(n_th: int):
    """The files READ_FLOW opens (for/diablo_io.f:208,232-236)."""
    return "diablo.start", [f"diablo_th{n + 1:02d}.start" for n in range(n_th)]


def _h5py():
    try:
        import h5py
    except ImportError as e:
        raise ImportError("HDF5 flow files need h5py; use save_flow/read_flow (unformatted) "
                          "or flow_fields_physical() with another HDF5 writer") from e
    return h5py


def write_h5(path: str, solver, final: bool = False):
    """WriteHDF5: end.h5 (final, with P) or out.h5 (no P)."""
    h5py = _h5py()
    p = solver.p
    d = solver.flow_fields_physical(pressure=final)
    t, _ = solver.get_time()
    with h5py.File(path, "w") as f:
        f.attrs["Resolution"] = [p.nx, p.ny, p.nz]
        f.attrs["Date"] = _time.strftime("%Y-%m-%d %H:%M:%S")
        f.attrs["Info"] = " (Put here what you want) "
        g = f.create_group("Timestep")
        g.attrs["Time"] = t
        for k, v in d.items():
            g.create_dataset(k, data=v, chunks=(v.shape[0], 1, v.shape[2]))


def read_h5(path: str, solver):
    """ReadHDF5: pressure if the file has it, else POISSON_P_CHAN."""
    h5py = _h5py()
    p = solver.p
    with h5py.File(path, "r") as f:
        res = list(f.attrs["Resolution"])
        if res != [p.nx, p.ny, p.nz]:
            raise ValueError(f"Error. File and program have different resolutions: {res}")
        g = f["Timestep"]
        d = {k: g[k][()] for k in g.keys()}
        t = float(g.attrs["Time"])
    solver.flow_fields_from_physical(d, t)
