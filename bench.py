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
single case is not sharded); value = all ranks' point-steps / max-over-ranks
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


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


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


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline(p, gy, seconds=15.0, threads=None):
    """Time the CPU oracle restatement (kind 'port') on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from diablo_b200 import ics
    threads = threads or os.cpu_count() or 1
    o = orc.Oracle(p, gy, threads=threads)
    u1, u2, u3, th = ics.channel_laminar(p, gy, seed=2)
    o.create_flow_chan(u1, u2, u3, th if p.n_th else None)
    o.set_time(0.0, p.delta_t)
    o.step(1)  # warm caches / plans
    t0 = time.perf_counter()
    n = 0
    while True:
        o.step(2 + n)
        n += 1
        if time.perf_counter() - t0 > seconds or n >= 50:
            break
    dt = time.perf_counter() - t0
    o.close()
    pts = p.nx * p.ny * p.nz
    return {"value": pts * n / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} full RK3 steps of the same 128x129x128 case (FP64 oracle, "
                      f"{threads} OpenMP threads, {dt:.1f} s)"}


def run_reference(args):
    """--impl reference: the oracle restatement on all host cores, rank 0 only."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from diablo_b200 import configs
    p, gy = configs.channel_re180()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from diablo_b200 import ics
    threads = os.cpu_count() or 1
    o = orc.Oracle(p, gy, threads=threads)
    u1, u2, u3, th = ics.channel_laminar(p, gy, seed=2)
    o.create_flow_chan(u1, u2, u3, None)
    o.set_time(0.0, p.delta_t)
    for s in range(args.warmup):
        o.step(1 + s)
    t0 = time.perf_counter()
    for s in range(args.steps):
        o.step(1 + args.warmup + s)
    dt = time.perf_counter() - t0
    o.close()
    pts = p.nx * p.ny * p.nz
    v = pts * args.steps / dt / 1e6
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(p),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} timed RK3 steps of the full case"},
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
        for rk in (1, 2, 3):
            ch.rk_chan_1(ts, rk)
        ch.advance_time()

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
    total = sum(times)
    if dist:
        t = torch.tensor([total], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    pts = p.nx * p.ny * p.nz
    value = ws * pts * args.steps / total / 1e6
    ms = 1e3 * total / args.steps

    # end to end through the C-ABI with host-owned state in the reference
    # layout (pinned host buffers), synced in and out every step
    names = ["CU1", "CU2", "CU3", "CP", "CF1", "CF2", "CF3"]
    refshape = (p.ny + 2, p.nz + 2, p.nx // 2 + 1)
    host = {n: torch.zeros(refshape + (2,), dtype=torch.float64).pin_memory() for n in names}
    for n in names:
        a = ch.get_field(n, layout="reference")
        host[n].numpy()[...] = np.stack([a.real, a.imag], -1)
    import ctypes
    L = _lib.load()
    e2e_steps = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for n in names:
            _lib.check("diablo_set_field", L.diablo_set_field(
                ch.h, _lib.field_id(n), ctypes.c_void_p(host[n].data_ptr()),
                _lib.DG_LAYOUT_REFERENCE, _lib.DG_HOST))
        ts += 1
        one_step(ts)
        for n in names:
            _lib.check("diablo_get_field", L.diablo_get_field(
                ch.h, _lib.field_id(n), ctypes.c_void_p(host[n].data_ptr()),
                _lib.DG_LAYOUT_REFERENCE, _lib.DG_HOST))
    ch.synchronize()
    e2e_t = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_t], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
    state_bytes = len(names) * int(np.prod(refshape)) * 16
    e2e = {"value": ws * pts * e2e_steps / e2e_t / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
           "steps": e2e_steps,
           "what": "per step: H2D of CU1..3, CP, CF1..3 in the reference layout from pinned "
                   "host memory, 3x diablo_rk_chan_1, D2H of the same fields"}

    # physical sanity of the timed run
    st = ch.stats()
    ch.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak, peak_kind = measured_peaks()
    bstep = algorithmic_bytes_per_step(p)
    achieved = bstep / (total / args.steps) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
            "scope": "whole RK3 step: algorithmic bytes (17 Nf + 6) x 16 B x M per step "
                     f"= {bstep / 1e6:.1f} MB over the device time of one step"}
    cpu = cpu_baseline(p, gy, seconds=args.cpu_seconds) if args.cpu_seconds > 0 else None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(p), "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clocks,
            "check": {"ke": st["ke"], "div_max": st["div_max"], "ubulk": st["ubulk"]}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
