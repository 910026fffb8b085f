"""Flow files (needs a B200): SAVE_FLOW / READ_FLOW in the reference's
unformatted layout and the arrays of its HDF5 flow files.

The expected bytes are built here with numpy from the reference's WRITE
statements (for/diablo_io.f:367-391): 4-byte record markers around a header
record (NX, NY, NZ, NUM_PER_DIR as int32, TIME as float64, TIME_STEP as
int32) and one record of retained modes.
"""
import struct

import numpy as np
import pytest

import oracle as O
from diablo_b200 import configs, ics, flow_io

pytestmark = pytest.mark.gpu


def rec(b: bytes) -> bytes:
    m = struct.pack("<i", len(b))
    return m + b + m


def header(p, time, ts):
    return rec(struct.pack("<4i", p.nx, p.ny, p.nz, p.num_per_dir) + struct.pack("<d", time)
               + struct.pack("<i", ts))


def channel_pair(p, gy, maker, seed, nsteps):
    from diablo_b200.solver import Channel
    ref = O.Oracle(p, gy)
    u1, u2, u3, th = maker(p, gy, seed=seed)
    ref.create_flow_chan(u1, u2, u3, th if p.n_th else None)
    ch = Channel(p, gy)
    ch.set_state(ref.state())
    ch.set_time(0.0, p.delta_t)
    for s in range(1, nsteps + 1):
        ch.step(s)
    return ref, ch


def test_save_flow_bytes_and_read_back(tmp_path):
    from diablo_b200.solver import Channel
    p, gy = configs.kh_shear_layer(nx=32, ny=17, nz=16)
    p = p.replace(n_th=2)
    p.ri = [0.1, 0.05, 0, 0]
    p.pr = [1.0, 0.7, 1, 1]
    _, ch = channel_pair(p, gy, ics.kh_shear_layer, seed=3, nsteps=3)
    fu, fth = flow_io.reference_names(False, p.n_th)
    fu, fth = str(tmp_path / fu), [str(tmp_path / f) for f in fth]
    ch.save_flow(fu, 3, fth)
    t, dt = ch.get_time()
    cu = {n: ch.get_field(n) for n in ("CU1", "CU2", "CU3", "CTH0", "CTH1")}
    ny = p.ny
    want = header(p, t, 3) + rec(cu["CU1"][1:ny + 1].tobytes() + cu["CU2"][2:ny + 1].tobytes()
                                 + cu["CU3"][1:ny + 1].tobytes())
    assert open(fu, "rb").read() == want
    for n in range(p.n_th):
        assert open(fth[n], "rb").read() == header(p, t, 3) + rec(cu[f"CTH{n}"][0:ny + 1].tobytes())

    fresh = Channel(p, gy)
    fresh.set_time(0.0, dt)
    ts = fresh.read_flow(fu, fth)
    assert ts == 3
    assert fresh.get_time()[0] == t
    # the planes outside the record start at zero, then APPLY_BC_VEL
    # (for/diablo_io.f:296-301) sets the ghost and wall planes
    exp = Channel(p, gy)
    st = {}
    for n, lo in (("CU1", 1), ("CU2", 2), ("CU3", 1)):
        a = np.zeros_like(cu[n])
        a[lo:ny + 1] = cu[n][lo:ny + 1]
        st[n] = a
    exp.set_state(st)
    exp.apply_bc_vel()
    for n in ("CU1", "CU2", "CU3"):
        assert np.array_equal(fresh.get_field(n), exp.get_field(n)), n
    exp.close()
    # scalars: written J=0..NY, read J=1..NY (for/diablo_io.f:379 vs :279)
    for n in range(p.n_th):
        a = fresh.get_field(f"CTH{n}")
        assert np.array_equal(a[1:ny + 1], cu[f"CTH{n}"][0:ny])
        assert not np.any(a[0]) and not np.any(a[ny + 1])
    # a file of other dimensions is refused with the reference's message
    q, gq = configs.kh_shear_layer(nx=32, ny=19, nz=16)
    other = Channel(q.replace(n_th=0), gq)
    with pytest.raises(Exception, match="wrong dimensions"):
        other.read_flow(fu)
    other.close()
    fresh.close()
    ch.close()


def test_periodic_flow_round_trip(tmp_path):
    from diablo_b200.solver import Periodic
    import math
    from diablo_b200.params import Params
    p = Params(nx=32, ny=32, nz=32, num_per_dir=3, nu=0.01, lx=2 * math.pi, ly=2 * math.pi,
               lz=2 * math.pi, delta_t=0.005, variable_dt=0)
    g = Periodic(p)
    for nm, a in zip(("CU1", "CU2", "CU3"), ics.periodic_spectrum(p, seed=4)):
        g.set_field(nm, a)
    g.set_time(0.25, p.delta_t)
    f = str(tmp_path / "diablo.saved")
    g.save_flow(f, 7)
    cu = {n: g.get_field(n) for n in ("CU1", "CU2", "CU3")}
    want = header(p, 0.25, 7) + rec(b"".join(cu[n].tobytes() for n in ("CU1", "CU2", "CU3")))
    assert open(f, "rb").read() == want
    h = Periodic(p)
    assert h.read_flow(f) == 7
    for n in ("CU1", "CU2", "CU3"):
        assert np.array_equal(h.get_field(n), cu[n])
    assert h.get_time()[0] == 0.25
    g.close()
    h.close()


def test_hdf5_dataset_arrays(tmp_path):
    from diablo_b200.solver import Channel
    p, gy = configs.channel_re180(nx=32, ny=33, nz=24)
    p = p.replace(variable_dt=0)
    ref, ch = channel_pair(p, gy, ics.channel_laminar, seed=5, nsteps=2)
    d = ch.flow_fields_physical(pressure=True)
    # expected: the physical fields (oracle transforms, the checker), V through
    # G2GF, then SWAPZY to [NZ][NY][NX] on planes 1..NY
    ny = p.ny
    phys = {n: ref.to_physical(ch.get_field(n)) for n in ("CU1", "CU2", "CU3", "CP")}
    v = phys["CU2"].copy()
    v[1] = v[2]
    v[ny + 1] = v[ny]
    for j in range(1, ny + 1):
        v[j] = 0.5 * (v[j] + v[j + 1])
    sw = lambda a: np.transpose(a[1:ny + 1], (1, 0, 2))
    for k, a in (("U", phys["CU1"]), ("V", v), ("W", phys["CU3"]), ("P", phys["CP"])):
        assert np.abs(d[k] - sw(a)).max() <= 1e-13 * np.abs(a).max(), k
    # ReadHDF5 of those arrays: U, W, P come back; V interior planes too, and
    # the walls are set for zero mass flux (V(1) = -V(2), V(NY+1) = -V(NY))
    cu = {n: ch.get_field(n) for n in ("CU1", "CU2", "CU3", "CP")}
    back = Channel(p, gy)
    back.flow_fields_from_physical(d, 0.5)
    assert back.get_time()[0] == 0.5
    for n in ("CU1", "CU3", "CP"):
        a, b = back.get_field(n)[1:ny + 1], cu[n][1:ny + 1]
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b), n
    a2 = back.get_field("CU2")
    assert np.linalg.norm(a2[2:ny + 1] - cu["CU2"][2:ny + 1]) <= 1e-12 * np.linalg.norm(cu["CU2"])
    assert np.linalg.norm(a2[1] + a2[2]) <= 1e-13 * np.linalg.norm(a2[2])
    # without P the pressure comes from POISSON_P_CHAN
    d.pop("P")
    nop = Channel(p, gy)
    nop.flow_fields_from_physical(d, 0.5)
    chk = Channel(p, gy)
    chk.set_state({n: back.get_field(n) for n in ("CU1", "CU2", "CU3")})
    chk.poisson_p_chan()
    a, b = nop.get_field("CP")[1:ny + 1], chk.get_field("CP")[1:ny + 1]
    assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)
    for s in (ch, back, nop, chk):
        s.close()
