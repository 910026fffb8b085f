"""Benchmark: DIABLO channel RK3/Crank-Nicolson step on B200.

Workload (the reference's Re_tau = 180 channel): 128 x 129 x 128 grid,
Lx = 4 pi, Ly = 2 (tanh stretch 1.75), Lz = 4 pi / 3, nu = 1/180, constant
pressure gradient, no-slip walls, CFL = 0.5 with COURANT every step, FP64.
Synthetic seeded initial condition (laminar parabola + Gaussian perturbation,
projected by REM_DIV_CHAN).  One "step" = three RK_CHAN_1 substeps + TIME
update.  Metric: Mpoint-steps/s = NX*NY*NZ per RK3 step.

  python bench.py [--gpus N --steps K --warmup W]      our sm_100a path
  python bench.py --impl reference ...                 CPU baseline: the FP64
                                                        oracle restatement of
                                                        RK_CHAN_1 on host cores

Under torchrun (N > 1) every rank advances its own independent replica (the
single case is not sharded), and the served ensemble deals whole cases out to
the ranks; value = all ranks' point-steps / max-over-ranks
time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

# the served ensemble runs one stream per active case: give the device more
# hardware work queues than the default 8 (read when the CUDA context starts)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK3 Mpoint-steps/s (channel Re_tau=180, FP64)"
UNIT = "Mpoint-steps/s"


def workload_config(p):
    return {"workload": "channel_re180_rk3_fp64", "nx": p.nx, "ny": p.ny, "nz": p.nz,
            "n_th": p.n_th, "cfl": p.cfl, "variable_dt": bool(p.variable_dt),
            "parallelism": "replicas", "l2": "flushed between timed steps (256 MiB write)"}


def algorithmic_bytes_per_step(p):
    """(17 Nf + 6) passes over one retained-mode FP64 field per RK3 step."""
    nf = 3 + p.n_th
    m = (p.nkx + 1) * (2 * p.nkz + 1) * (p.ny + 2)
    return (17 * nf + 6) * 16 * m


def kernel_bytes_per_launch(p, name):
    """Algorithmic HBM bytes of one launch of a channel-substep kernel: each
    array the kernel must read or write, once (stencil neighbours and halo
    rows are free).  Fields are FP64 complex (16 B); the REM_DIV factors are
    FP64 real.  CF_old is read in substeps 2 and 3 only: counted at 2/3.
    M: retained modes x all planes; Si: x interior planes; Mh, Mi: half-
    physical values (NZ x (NKX+1) per plane) on all / interior planes."""
    nf = 3 + p.n_th
    th_copies = sum(1 for n in range(p.n_th)
                    if p.ri[n] * p.grav_x != 0 or p.ri[n] * p.grav_y != 0
                    or p.ri[n] * p.grav_z != 0)
    nkxp, nkzt = p.nkx + 1, 2 * p.nkz + 1
    L, NY, NZ = p.ny + 2, p.ny, p.nz
    ss = nkxp * nkzt
    M, Si = ss * L, ss * NY                 # spectral values, all / interior planes
    Mh, Mi = L * NZ * nkxp, NY * NZ * nkxp  # half-physical values, all / interior planes
    c = 16
    table = {
        "k_zinv": c * nf * (M + Mh),
        "k_xrow_w": c * (nf * Mh + 2 * nf * Mi),
        # z forward of the 2 Nf product arrays; writes NL of every field
        "k_zfwd_w": c * (2 * nf * Mi + nf * Si),
        # column stage, all fields: read CU, NL, CF_old and CP (once); write
        # CF and the post-CN field
        "k_col_cn": c * (2 * nf * M + nf * Si * (1 + 2 / 3 + 1) + M),
        # REM_DIV from the post-CN velocity: read U and CP, write U, phi and
        # CP, read the two factor arrays; copy the scalars that a velocity
        # right-hand side reads (left in the rhs arrays) into CU
        "k_rd_col": c * (4 * M + 5 * M) + 8 * 2 * M + c * 2 * M * th_copies,
        "k_xc2r_cfl": c * 3 * Mh,
    }
    return table.get(name)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` (dram__bytes_read.sum +
    dram__bytes_write.sum) from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic_channel_re180.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel:
                    return float(parts[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except Exception:
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.out.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def replica_throughput(dist, ws, seconds, pts_per_step, steps, device="cuda"):
    """Whole-job Mpoint-steps/s of ws independent replicas: every rank did
    `steps` steps of `pts_per_step` points in `seconds` of its own device
    time; the job took as long as the slowest rank (max over ranks)."""
    if dist is not None:
        import torch
        t = torch.tensor([seconds], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        seconds = float(t.item())
    return ws * pts_per_step * steps / seconds / 1e6, seconds


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def host_cpus():
    """Host threads this process may use, and what the host is: the CPU
    affinity set (what nproc reports), capped by a cgroup CPU quota where one
    is set; physical cores in that set; the CPU model; the load average."""
    try:
        allowed = sorted(os.sched_getaffinity(0))
    except Exception:
        allowed = list(range(os.cpu_count() or 1))
    quota = None
    try:
        q, per = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if q != "max":
            quota = float(q) / float(per)
    except Exception:
        pass
    threads = len(allowed)
    if quota:
        threads = max(1, min(threads, int(quota + 0.5)))
    model, cores = None, set()
    try:
        cpu, phys, core = None, None, None
        for line in open("/proc/cpuinfo"):
            k, _, v = line.partition(":")
            k, v = k.strip(), v.strip()
            if k == "processor":
                cpu = int(v)
            elif k == "model name" and model is None:
                model = v
            elif k == "physical id":
                phys = v
            elif k == "core id":
                core = v
            elif not k and cpu is not None:
                if cpu in allowed:
                    cores.add((phys, core))
                cpu = phys = core = None
    except Exception:
        pass
    try:
        load = os.getloadavg()[0]
    except Exception:
        load = None
    return {"threads": threads, "nproc": len(allowed), "cpu_count": os.cpu_count(),
            "physical_cores": len(cores) or None, "cgroup_cpu_quota": quota,
            "cpu_model": model, "loadavg_1min": load}


def time_oracle(p, gy, warmup, steps, max_seconds=60.0):
    """Time the CPU oracle restatement of RK_CHAN_1 (kind 'port') on this
    host: `warmup` untimed RK3 steps, then up to `steps` timed ones (fewer if
    `max_seconds` runs out), each timed on its own; the figure is the median
    step.  Both CPU legs of the benchmark (the reference arm and the
    cpu_baseline record) call this with the same warm-up and step count.
    OpenMP threads are pinned one per allowed CPU, packed by core
    (OMP_PROC_BIND=close, OMP_PLACES=cores, unless the caller set them), so
    the thread placement does not change between runs."""
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from diablo_b200 import ics
    host = host_cpus()
    threads = host["threads"]
    o = orc.Oracle(p, gy, threads=threads)
    u1, u2, u3, th = ics.channel_laminar(p, gy, seed=2)
    o.create_flow_chan(u1, u2, u3, th if p.n_th else None)
    o.set_time(0.0, p.delta_t)
    for s in range(warmup):
        o.step(1 + s)
    per = []
    t0 = time.perf_counter()
    for s in range(steps):
        a = time.perf_counter()
        o.step(1 + warmup + s)
        per.append(time.perf_counter() - a)
        if time.perf_counter() - t0 > max_seconds:
            break
    o.close()
    med = statistics.median(per)
    pts = p.nx * p.ny * p.nz
    spread = (min(per), max(per))
    return {"value": pts / med / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "ms_per_step_median": 1e3 * med,
            "ms_per_step_min_max": [1e3 * spread[0], 1e3 * spread[1]],
            "host": host,
            "omp": {k: os.environ.get(k) for k in ("OMP_PROC_BIND", "OMP_PLACES")},
            "sample": f"median of {len(per)} timed RK3 steps (after {warmup} untimed) of the full "
                      f"{p.nx}x{p.ny}x{p.nz} case, FP64 oracle on {threads} OpenMP threads"}


def cpu_baseline(p, gy, warmup=5, steps=20):
    """The cpu_baseline record: the same measurement as the reference arm."""
    return time_oracle(p, gy, warmup, steps)


def run_ensemble(args, dist=None, ws=1, rank=0):
    """The served-ensemble workload: KH cases with NX in {64,128,256}, NZ in
    {16,32,64}, NY in {33,65,129} (uniform on [-10,10]), Re ~ U[500,5000],
    Ri ~ U[0.05,0.25], seeded 1e-3 noise, Poisson arrivals at `rate`/s, each
    run for `steps` RK3 steps in mixed precision under a 150 GB budget through
    the continuous-batching server (grouped stepping with ragged column
    launches, and every case on its own stream).  Beside it, the plain
    per-case FP64 path (one case at a time, graph-replayed steps) over the
    same workload: every grid shape timed alone.
    Under torchrun every rank serves the cases the host-side dispatcher gives
    it (whole cases, no data exchanged) and the ranks pool their statistics."""
    import torch
    from diablo_b200 import configs, ics
    from diablo_b200.grid import uniform_grid
    from diablo_b200.serve import Server, assign_cases, merge_rank_stats
    from diablo_b200.solver import Channel
    rng = np.random.default_rng(5)
    base, _ = configs.kh_shear_layer()
    cases = []
    for _ in range(args.ensemble_cases):
        q = ics.ensemble_kh_params(rng, base)
        cases.append((q, uniform_grid(q.ny, -10.0, 10.0)))
    arrivals = np.cumsum(rng.exponential(1.0 / args.ensemble_rate, len(cases)))
    mine = [i for i, r in enumerate(assign_cases(
        [q.nx * q.ny * q.nz * args.ensemble_steps for q, _ in cases], ws)) if r == rank]
    # plain per-case FP64 path, size-stratified: every one of the 27 grid
    # shapes timed alone (graph-replayed steps, device time), then the plain
    # time of the whole workload is the sum over the cases of their shape's
    # step time (the step cost does not depend on Re or Ri at fixed dt)
    shape_ms = {}
    psteps = min(args.ensemble_steps, 100)
    if rank == 0:
        for nx in (64, 128, 256):
            for ny in (33, 65, 129):
                for nz in (16, 32, 64):
                    q = base.replace(nx=nx, ny=ny, nz=nz)
                    gy = uniform_grid(ny, -10.0, 10.0)
                    st = torch.cuda.Stream()
                    ch = Channel(q, gy, stream=st.cuda_stream)
                    for k, v in ics.kh_state(q, gy, seed=7).items():
                        ch.set_field(k, v)
                    ch.set_time(0.0, q.delta_t)
                    ch.apply_bc_vel()
                    ch.rem_div_chan()
                    ch.apply_bc_vel()
                    ch.steps(1, 3)
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    ch.steps(4, psteps)
                    e1.record(st)
                    e1.synchronize()
                    shape_ms[(nx, ny, nz)] = e0.elapsed_time(e1) / psteps
                    ch.close()
    plain = None
    if shape_ms:
        pts = sum(q.nx * q.ny * q.nz for q, _ in cases)
        secs = sum(shape_ms[(q.nx, q.ny, q.nz)] * 1e-3 for q, _ in cases)
        plain = pts / secs / 1e6

    def serve(group):
        # served, mixed precision, continuous batching; every rank starts its
        # clock together so the shared arrival process lines up across ranks
        if dist:
            dist.barrier()
        srv = Server(max_active=args.ensemble_active, budget_gb=150.0, autotune=True,
                     group_cases=group)
        t0 = time.perf_counter()
        ids = []
        for i in mine:
            q, gy = cases[i]
            st0 = ics.kh_state(q, gy, seed=100 + i)
            delay = t0 + arrivals[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(q.replace(precision=1), gy, st0, args.ensemble_steps))
        lat = []
        for cid in ids:
            _, (qs, rs) = srv.wait(cid)
            lat.append(qs + rs)
        wall = time.perf_counter() - t0
        s = srv.stats()
        srv.close()
        rec = {"wall_s": s["wall_s"] if mine else 0.0, "cases": len(mine),
               "points": sum(cases[i][0].nx * cases[i][0].ny * cases[i][0].nz for i in mine)
               * args.ensemble_steps,
               "case_latency_s": lat, "step_ms_p50": s["step_ms_p50"], "step_ms_p99": s["step_ms_p99"],
               "hbm_peak_gb": s["bytes_peak"] / 1e9}
        if dist:
            allrec = [None] * ws
            dist.all_gather_object(allrec, rec)
        else:
            allrec = [rec]
        m = merge_rank_stats(allrec)
        out = {"cases_per_s": m["cases_per_s"], "step_ms_p50": m["step_ms_p50_worst_rank"],
               "step_ms_p99": m["step_ms_p99_worst_rank"],
               "mpoint_steps_per_s": m["mpoint_steps_per_s"],
               "case_latency_s_p50": m["case_latency_s_p50"],
               "case_latency_s_p99": m["case_latency_s_p99"],
               "hbm_peak_gb": m["hbm_peak_gb_max"], "wall_s": wall}
        if plain and ws == 1:
            out["served_over_plain"] = m["mpoint_steps_per_s"] / plain
        elif plain:
            out["served_per_gpu_over_plain"] = m["mpoint_steps_per_s"] / ws / plain
        return out

    grouped = serve(args.ensemble_group)
    alone = serve(0) if args.ensemble_group else None
    out = {"cases": len(cases), "steps_per_case": args.ensemble_steps,
           "arrival_rate_per_s": args.ensemble_rate, "max_active": args.ensemble_active,
           "gpus": ws, "dispatch": "whole cases per GPU, longest first to the least-loaded GPU",
           "precision": "mixed (FP32 transforms and products, FP64 solves)",
           "group_cases": args.ensemble_group,
           "stepping": (f"groups of up to {args.ensemble_group} cases of similar size, one graph "
                        "per group step, one ragged column launch per substep"
                        if args.ensemble_group else "every case on its own stream"),
           "plain_fp64_mpoint_steps_per_s": plain,
           "plain_sample": (f"all 27 grid shapes alone on one GPU, {psteps} FP64 steps each; "
                            "the workload's plain time is the sum over its cases of their "
                            "shape's step time"),
           "plain_shape_ms_per_step": {f"{a}x{b}x{c}": round(v, 4)
                                       for (a, b, c), v in sorted(shape_ms.items())}}
    out.update(grouped)
    if alone is not None:
        out["per_case_streams"] = alone
    return out


def step_timer(ts):
    """ms per full step over graph-replayed steps on stream ts (CUDA events,
    L2 not flushed), after `warm` untimed steps."""
    import torch

    def timed(solver, nsteps, warm=3):
        solver.steps(1, warm)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ts)
        solver.steps(warm + 1, nsteps)
        e1.record(ts)
        e1.synchronize()
        return e0.elapsed_time(e1) / nsteps
    return timed


LES_CASES = {"kh_les": "kh_les_128x65x16", "channel_re180_les": "channel_re180_les_128x129x128",
             "channel_re180_les_mixed": "channel_re180_les_128x129x128_mixed"}


def run_les_configs(ts, timed, nsteps, cpu=True, only=""):
    """LES (constant Smagorinsky, FP64): the reference's KH_test run and the
    Re_tau = 180 channel with the model on, each timed over nsteps
    graph-replayed steps; the CPU oracle's time for the KH_test step beside it
    (all host threads, 2 steps)."""
    from diablo_b200 import configs, ics
    from diablo_b200.solver import Channel
    stream = ts.cuda_stream
    out = {}
    p180, gy180 = configs.channel_re180()
    for name, (p, gy), maker in (("kh_les_128x65x16", configs.kh_les(), ics.kh_shear_layer),
                                 ("channel_re180_les_128x129x128",
                                  (p180.replace(les=1), gy180), ics.channel_laminar),
                                 ("channel_re180_les_128x129x128_mixed",
                                  (p180.replace(les=1, precision=1), gy180), ics.channel_laminar)):
        if only and name != LES_CASES[only]:
            continue
        kw = {"kick": 0.1} if maker is ics.kh_shear_layer else {}
        u1, u2, u3, th = maker(p, gy, seed=2, **kw)
        ch = Channel(p, gy, stream=stream)
        ch.create_flow(u1, u2, u3, th if p.n_th else None)
        ch.set_time(0.0, p.delta_t)
        ms = timed(ch, nsteps)
        rec = {"ms_per_step": ms, "mpoint_steps_per_s": p.nx * p.ny * p.nz / ms / 1e3,
               "nu_t_max": float(ch.nu_t().max())}
        ch.close()
        if cpu and name.startswith("kh_les"):
            import oracle as O
            ref = O.Oracle(p, gy, threads=os.cpu_count() or 1)
            ref.create_flow_chan(u1, u2, u3, th)
            t0 = time.perf_counter()
            for s in (1, 2):
                ref.step(s)
            rec["cpu_baseline"] = {"ms_per_step": (time.perf_counter() - t0) / 2 * 1e3,
                                   "cores": os.cpu_count() or 1, "kind": "port",
                                   "sample": "2 steps of the same case"}
            ref.close()
        out[name if p.precision else name + "_fp64"] = rec
    return out


def run_other_configs(args):
    """The other configurations of the workload list, each timed for a few
    graph-replayed steps (CUDA events, L2 not flushed): FP64 and mixed where
    both exist.  Parity for each is in the test suite."""
    import torch
    from diablo_b200 import configs, ics
    from diablo_b200.solver import Channel, Periodic

    ts = torch.cuda.Stream()     # the solvers run on this stream; events are recorded on it
    stream = ts.cuda_stream
    timed = step_timer(ts)
    out = {}

    def errors(fin, names, stats):
        """The mixed run against the FP64 run from the same state over the same
        steps: per-field relative L2, and both runs' max |div u|."""
        return {"rel_l2_vs_fp64_gpu": {nm: float(np.linalg.norm(fin[1][nm] - fin[0][nm])
                                                 / np.linalg.norm(fin[0][nm])) for nm in names},
                "div_max": {"fp64": stats[0]["div_max"], "mixed": stats[1]["div_max"]}}

    # KH shear layer 128 x 65 x 32 and Re_tau = 180, FP64 and mixed
    for name, (p, gy), maker in (("kh_shear_layer_128x65x32", configs.kh_shear_layer(),
                                  ics.kh_shear_layer),
                                 ("channel_re180_128x129x128", configs.channel_re180(),
                                  ics.channel_laminar)):
        names = ["CU1", "CU2", "CU3"] + [f"CTH{n}" for n in range(p.n_th)]
        fin, stats, growth = {}, {}, {}
        for prec in (0, 1):
            ch = Channel(p.replace(precision=prec), gy, stream=stream)
            u1, u2, u3, th = maker(p, gy, seed=2)
            ch.create_flow(u1, u2, u3, th if p.n_th else None)
            ch.set_time(0.0, p.delta_t)
            start = ch.get_state()
            ch.autotune(2)
            ms = timed(ch, 100)
            fin[prec] = {nm: ch.get_field(nm) for nm in names}
            stats[prec] = ch.stats()
            if name.startswith("kh"):
                # growth rate of the vertical-velocity energy over 100 steps
                # from the seeded state (least squares on ln <v^2>, every 10)
                ch.set_state(start)
                ch.set_time(0.0, p.delta_t)
                t, e2 = [], []
                for k in range(10):
                    ch.steps(1 + 10 * k, 10)
                    t.append(10 * (k + 1) * p.delta_t)
                    e2.append(ch.stats()["vrms_b"] ** 2)
                growth[prec] = float(np.polyfit(t, np.log(e2), 1)[0])
            ch.close()
            out[f"{name}_{'mixed' if prec else 'fp64'}"] = {
                "ms_per_step": ms, "mpoint_steps_per_s": p.nx * p.ny * p.nz / ms / 1e3}
        rec = errors(fin, names, stats)
        rec["after_steps"] = 103
        if growth:
            rec["kh_growth_rate"] = {"fp64": growth[0], "mixed": growth[1],
                                     "rel_err": abs(growth[1] - growth[0]) / abs(growth[0])}
        out[f"{name}_mixed"]["error"] = rec
    out.update(run_les_configs(ts, timed, 50))
    # periodic 256^3, FP64 and mixed from the same state over the same steps
    p, _ = configs.periodic_256()
    fin, stats = {}, {}
    for prec in (0, 1):
        g = Periodic(p.replace(precision=prec), stream=stream)
        for nm, a in zip(("CU1", "CU2", "CU3"), ics.periodic_spectrum(p, seed=3)):
            g.set_field(nm, a)
        g.set_time(0.0, p.delta_t)
        g.rem_div_per()
        g.poisson_p_per()
        ms = timed(g, 20)
        fin[prec] = {nm: g.get_field(nm) for nm in ("CU1", "CU2", "CU3")}
        stats[prec] = g.stats()
        g.close()
        out[f"periodic_256cubed_{'mixed' if prec else 'fp64'}"] = {
            "ms_per_step": ms, "mpoint_steps_per_s": 256 ** 3 / ms / 1e3}
    rec = errors(fin, ("CU1", "CU2", "CU3"), stats)
    rec["after_steps"] = 23
    out["periodic_256cubed_mixed"]["error"] = rec
    # Re_tau ~ 550, 512 x 257 x 384, one scalar: FP64 and mixed from the same
    # state, each timed over the same steps
    p, gy = configs.channel_re550()
    u1, u2, u3, th = ics.channel_laminar(p, gy, seed=4)
    fin, stats = {}, {}
    for prec in (0, 1):
        ch = Channel(p.replace(precision=prec), gy, stream=stream)
        if prec == 0:
            ch.create_flow(u1, u2, u3, th)
            start = ch.get_state()
        else:
            ch.set_state(start)
        ch.set_time(0.0, p.delta_t)
        ms = timed(ch, 10, warm=3)
        fin[prec] = {nm: ch.get_field(nm) for nm in ("CU1", "CU2", "CU3", "CTH0")}
        stats[prec] = ch.stats()
        ch.close()
        out[f"channel_re550_512x257x384_{'mixed' if prec else 'fp64'}"] = {
            "ms_per_step": ms, "mpoint_steps_per_s": p.nx * p.ny * p.nz / ms / 1e3}
    rec = errors(fin, ("CU1", "CU2", "CU3", "CTH0"), stats)
    rec["after_steps"] = 13
    out["channel_re550_512x257x384_mixed"]["error"] = rec
    out["mixed_error_note"] = (
        "error records compare each mixed run with the FP64 GPU run from the same state over "
        "the same steps; the FP64 GPU path is itself held to 1e-11 of the FP64 oracle, and "
        "the mixed runs to 1e-5 of the oracle directly, by the GPU tests (100 steps KH and "
        "Re_tau=180, 200 steps periodic 256^3, 10 steps Re_tau~550 at full size)")
    return out


def run_reference(args):
    """--impl reference: the oracle restatement on all host cores, rank 0 only."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from diablo_b200 import configs
    p, gy = configs.channel_re180()
    # bounded sample: at most 200 timed steps, at most 120 s of them
    rec = time_oracle(p, gy, args.warmup, min(args.steps, 200), max_seconds=120.0)
    v = rec["value"]
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": rec["ms_per_step_median"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference", "config": workload_config(p),
            "cpu_baseline": rec,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_gpu(args):
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from diablo_b200 import _lib, configs, ics
    from diablo_b200.solver import Channel

    p, gy = configs.channel_re180()
    stream = torch.cuda.Stream()
    ch = Channel(p, gy, stream=stream.cuda_stream)
    u1, u2, u3, _ = ics.channel_laminar(p, gy, seed=2 + rank)
    ch.create_flow(u1, u2, u3)
    ch.set_time(0.0, p.delta_t)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def one_step(ts):
        # diablo_step: the driver's loop body; CUDA-graph replay after the
        # first step of each kind
        ch.steps(ts, 1)

    def one_step_eager(ts):
        for rk in (1, 2, 3):
            ch.rk_chan_1(ts, rk)
        ch.advance_time()

    # launch shapes: the library's autotuner times candidates on this state
    # and restores it (part of set-up, outside the timed region); --tuning
    # fixes them instead (for profiling runs that must not time the tuner)
    if args.tuning:
        ch.tune_set(**{k: int(v) for k, v in (kv.split("=") for kv in args.tuning.split(","))})
        tuned = ch.tune_get()
    else:
        tuned = ch.autotune(3)
    ts = 0
    for _ in range(args.warmup):
        ts += 1
        one_step(ts)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    L = _lib.load()
    launches0 = _lib.kernel_launches()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)  # evict L2 (outside the timed region)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            stream.wait_stream(torch.cuda.current_stream())
            e0.record(stream)
            ts += 1
            one_step(ts)
            e1.record(stream)
        torch.cuda.current_stream().wait_stream(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    torch.cuda.synchronize()
    launches = _lib.kernel_launches() - launches0
    clocks = sampler.stop() if sampler else None
    # per-kernel device times: CUDA events around every launch of the same
    # step run eagerly (graph replays carry no per-kernel events), right after
    # the timed region, L2 flushed between steps as above
    kt_steps = max(3, min(args.steps, 100))
    _lib.check("dg_timing_enable", L.dg_timing_enable(ch.h, 1))
    for _ in range(kt_steps):
        flush.fill_(1.0)
        stream.wait_stream(torch.cuda.current_stream())
        ts += 1
        one_step_eager(ts)
        torch.cuda.current_stream().wait_stream(stream)
    torch.cuda.synchronize()
    _lib.check("dg_timing_enable", L.dg_timing_enable(ch.h, 0))
    kt = {}
    import ctypes
    nm = ctypes.create_string_buffer(64)
    cnt = ctypes.c_int64()
    tms = ctypes.c_double()
    i = 0
    while L.dg_timing_read(ch.h, i, nm, 64, ctypes.byref(cnt), ctypes.byref(tms)) == 0:
        kt[nm.value.decode()] = (int(cnt.value), float(tms.value))
        i += 1
    pts = p.nx * p.ny * p.nz
    value, total = replica_throughput(dist, ws, sum(times), pts, args.steps)
    ms = 1e3 * total / args.steps

    # end to end through the C-ABI with host-owned state in the reference
    # layout (pinned host buffers), synced in and out every step
    # a step reads CU1..3 and CP (CF is rebuilt by substep 1 before use) and
    # returns the same fields
    names = ["CU1", "CU2", "CU3", "CP"] + [f"CTH{n}" for n in range(p.n_th)]
    refshape = (p.ny + 2, p.nz + 2, p.nx // 2 + 1)
    host = {n: torch.zeros(refshape + (2,), dtype=torch.float64).pin_memory() for n in names}
    for n in names:
        a = ch.get_field(n, layout="reference")
        host[n].numpy()[...] = np.stack([a.real, a.imag], -1)
    e2e_steps = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ids = (ctypes.c_int * len(names))(*[_lib.field_id(n) for n in names])
    ptrs = (ctypes.c_void_p * len(names))(*[host[n].data_ptr() for n in names])
    for _ in range(e2e_steps):
        _lib.check("diablo_set_fields", L.diablo_set_fields(
            ch.h, len(names), ids, ptrs, _lib.DG_LAYOUT_REFERENCE_RETAINED, _lib.DG_HOST))
        ts += 1
        one_step(ts)
        _lib.check("diablo_get_fields", L.diablo_get_fields(
            ch.h, len(names), ids, ptrs, _lib.DG_LAYOUT_REFERENCE_RETAINED, _lib.DG_HOST))
    ch.synchronize()
    e2e_value, e2e_t = replica_throughput(dist, ws, time.perf_counter() - t0, pts, e2e_steps)
    # bytes that cross the bus: set_field and get_field copy the retained
    # block of each reference array (kx 0..NKX, packed kz 0..TNKZ, all
    # planes), one strided copy each way
    retained = (p.ny + 2) * (2 * (p.nz // 3) + 1) * (p.nx // 3 + 1)
    h2d_bytes = len(names) * retained * 16
    d2h_bytes = len(names) * retained * 16
    e2e = {"value": e2e_value, "unit": UNIT,
           "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
           "steps": e2e_steps,
           "what": "per step: H2D of CU1..3 and CP from reference-layout pinned host arrays "
                   "(diablo_set_fields: the retained block, one strided copy each, on two "
                   "streams), one diablo_step (3 RK_CHAN_1 substeps + TIME update), D2H of the "
                   "same fields' retained block into the reference-layout arrays "
                   "(diablo_get_fields, REFERENCE_RETAINED)"}

    # physical sanity of the timed run
    st = ch.stats()
    ch.close()
    ens = run_ensemble(args, dist, ws, rank) if args.ensemble_cases > 0 else None
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak, peak_kind = measured_peaks()
    bstep = algorithmic_bytes_per_step(p)
    step_achieved = bstep / (total / args.steps) / 1e9
    # dominant kernel: largest share of the event-timed device time
    dom = max(kt.items(), key=lambda kv: kv[1][1]) if kt else None
    roof = None
    if dom is not None:
        name, (n, ms_tot) = dom
        per = kernel_bytes_per_launch(p, name)
        avg_s = ms_tot * 1e-3 / max(n, 1)
        achieved = per / avg_s / 1e9 if per else None
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "traffic": ncu_traffic(name), "bytes_per_launch": per,
                "avg_launch_us": avg_s * 1e6, "launches": n,
                "share": ms_tot / sum(v[1] for v in kt.values()),
                "timing": f"CUDA events around each launch over {kt_steps} eager steps run right "
                          "after the timed region (same kernels as the graph replays)",
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                else "fallback 6650 GB/s"}
    kernels = {k: {"launches": v[0], "total_ms": round(v[1], 3),
                   "avg_us": round(1e3 * v[1] / max(v[0], 1), 2)} for k, v in kt.items()}
    roof_step = {"achieved": step_achieved, "peak": peak, "unit": "GB/s",
                 "frac": step_achieved / peak,
                 "scope": "whole RK3 step: algorithmic bytes (17 Nf + 6) x 16 B x M per step "
                          f"= {bstep / 1e6:.1f} MB over the device time of one step"}
    cpu = cpu_baseline(p, gy) if args.cpu_seconds > 0 else None
    others = run_other_configs(args) if args.other_configs else None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(p), tuning=tuned), "roofline": roof, "roofline_step": roof_step,
            "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e, "ensemble": ens,
            "other_configs": others,
            "gpu_launches": int(launches), "clocks": clocks,
            "check": {"ke": st["ke"], "div_max": st["div_max"], "ubulk": st["ubulk"]}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="0 skips the cpu_baseline record (5 untimed + 20 timed oracle steps)")
    ap.add_argument("--tuning", default="",
                    help="fixed launch shapes, e.g. col_mt=8,cn_mt=16,xrow_chunk=0,ychunk=0")
    ap.add_argument("--other-configs", type=int, default=1,
                    help="also time the other workload configurations (0 = skip)")
    ap.add_argument("--ensemble-cases", type=int, default=256)
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--ensemble-rate", type=float, default=20.0)
    ap.add_argument("--ensemble-active", type=int, default=16)
    ap.add_argument("--ensemble-group", type=int, default=4,
                    help="cases per step group in the served ensemble (0: every case alone)")
    ap.add_argument("--les-only", default="", choices=["", "all"] + list(LES_CASES),
                    help="time only the LES workloads (all, or the one named; --steps "
                         "graph-replayed steps each, after --warmup) and print their records; "
                         "no contract line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.les_only:
        import torch
        ts = torch.cuda.Stream()
        timed = step_timer(ts)
        out = run_les_configs(ts, lambda ch, n: timed(ch, n, warm=args.warmup), args.steps,
                              cpu=False, only="" if args.les_only == "all" else args.les_only)
        print(json.dumps({"les": out}))
        return 0
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
