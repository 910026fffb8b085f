"""The N > 1 plumbing of bench.py on CPU: two gloo ranks (the single case
does not shard; every rank runs a replica and the job takes as long as the
slowest rank), and the reference arm's rank-0-only rule."""
import os
import socket
import subprocess
import sys

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
