"""bench.py's multi-rank aggregation (barrier, max of the device times, sum of the lattice updates) as two gloo
ranks on CPU: every rank gets the same max and sum, as rank 0 reports them."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, str(ROOT))
    import bench
    bench.barrier(world)
    ms = bench.max_over_ranks(10.0 + rank, world)  # per-rank device time
    lups = bench.sum_over_ranks(1000.0 * (rank + 1), world)  # per-rank lattice updates
    q.put((rank, ms, lups))
    dist.destroy_process_group()


def test_rank_aggregation_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 11.0, 3000.0), (1, 11.0, 3000.0)]
