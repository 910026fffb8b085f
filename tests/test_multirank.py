"""The N > 1 plumbing of bench.py on CPU: two gloo ranks (the single case
does not shard; every rank runs a replica and the job takes as long as the
slowest rank), and the reference arm's rank-0-only rule."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    # rank r spent 1 + r seconds on 10 steps of 1e6 points
    value, secs = bench.replica_throughput(dist, ws, 1.0 + rank, 1_000_000, 10, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, value, secs))


def test_replica_throughput_is_max_over_ranks():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, secs in res:
        assert secs == 2.0                      # the slowest rank's time, on every rank
        assert abs(value - ws * 1e6 * 10 / 2.0 / 1e6) < 1e-9


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""               # ranks other than 0 print nothing


def test_assign_cases_balances_whole_cases():
    from diablo_b200.serve import assign_cases
    rng = np.random.default_rng(3)
    work = list(rng.integers(1, 1000, size=257))
    for world in (1, 2, 3, 8):
        r = assign_cases(work, world)
        assert len(r) == len(work) and set(r) <= set(range(world))
        assert r == assign_cases(work, world)            # every rank computes the same
        load = np.bincount(r, weights=work, minlength=world)
        assert load.max() - load.min() <= max(work)      # LPT bound
    assert assign_cases([5.0, 5.0], 4) == [0, 1]


def test_merge_rank_stats():
    from diablo_b200.serve import merge_rank_stats
    a = {"wall_s": 2.0, "cases": 3, "points": 6e6, "case_latency_s": [1.0, 2.0, 3.0],
         "step_ms_p50": 1.0, "step_ms_p99": 4.0, "hbm_peak_gb": 1.5}
    b = {"wall_s": 4.0, "cases": 1, "points": 2e6, "case_latency_s": [5.0],
         "step_ms_p50": 2.0, "step_ms_p99": 3.0, "hbm_peak_gb": 0.5}
    m = merge_rank_stats([a, b])
    assert m["wall_s"] == 4.0 and m["cases"] == 4
    assert m["cases_per_s"] == 1.0 and m["mpoint_steps_per_s"] == 2.0
    assert m["step_ms_p50_worst_rank"] == 2.0 and m["step_ms_p99_worst_rank"] == 4.0
    assert m["case_latency_s_p50"] == 2.5 and m["hbm_peak_gb_max"] == 1.5


def _ens_rank(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from diablo_b200.serve import assign_cases, merge_rank_stats
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    work = [(i % 7 + 1) * 1000 for i in range(20)]
    mine = [i for i, r in enumerate(assign_cases(work, ws)) if r == rank]
    rec = {"wall_s": 1.0 + rank, "cases": len(mine), "points": float(sum(work[i] for i in mine)),
           "case_latency_s": [float(i) for i in mine], "step_ms_p50": 1.0, "step_ms_p99": 2.0,
           "hbm_peak_gb": 0.1}
    allrec = [None] * ws
    dist.all_gather_object(allrec, rec)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, merge_rank_stats(allrec)))


def test_ensemble_dispatch_over_two_gloo_ranks():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ens_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in range(ws)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = sorted(res[0][1] + res[1][1])
    assert got == list(range(20))                      # every case on exactly one rank
    m0, m1 = res[0][2], res[1][2]
    assert m0 == m1                                    # both ranks pool the same figures
    work = [(i % 7 + 1) * 1000 for i in range(20)]
    assert m0["wall_s"] == 2.0 and m0["cases"] == 20
    assert abs(m0["mpoint_steps_per_s"] - sum(work) / 2.0 / 1e6) < 1e-12
