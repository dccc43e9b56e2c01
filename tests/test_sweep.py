"""Design sharding and the result gather of xadvcool_b200.sweep, on CPU: world_size 2 over gloo, with the
per-design solve replaced by the CPU oracle (the sharding/gather logic is what is under test)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from xadvcool_b200 import sweep


def test_shard_is_a_balanced_partition():
    costs = [5, 1, 9, 3, 3, 7, 2, 8]
    for world in (1, 2, 3, 8, 11):
        parts = sweep.shard(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert sweep.shard(costs, 2) == sweep.shard(costs, 2)  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_solver(designs, indices, **kw):
    from oracle.ref import Ref
    rows = []
    for i in indices:
        d = designs[i]
        r = Ref(32).run_simulation(d["mask"], max_steps=60, tau_fluid=d["tau_fluid"], u_inlet_val=d["u_inlet_val"],
                                   tol_ke=0, tol_T=0)
        rows.append([i, r["steps"], r["converged"], r["diverged"], float(r["rho"].mean()), float(r["T"].max()),
                     float(np.abs(r["u"]).max()), 0, 0, 0, 0, 0])
    return np.asarray(rows, dtype=np.float64).reshape(-1, len(sweep.RESULT_COLS))


def _designs():
    rng = np.random.default_rng(0)
    out = []
    for k in range(5):
        nx = 8 + 2 * k
        m = np.zeros((nx, 6, 5), np.int32)
        m[:, 0] = 1
        m[:, -1] = 1
        m[rng.random(m.shape) < 0.1] = 1
        m[0, 1:-1, 1:-1] = 2
        m[-1, 1:-1, 1:-1] = 3
        out.append(dict(mask=m, tau_fluid=0.6 + 0.01 * k, u_inlet_val=0.02))
    return out


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        table = sweep.run_sweep(_designs(), rank=rank, world=world, solver=_oracle_solver)
        q.put((rank, table))
    finally:
        dist.destroy_process_group()


def test_two_rank_sweep_matches_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    single = sweep.run_sweep(_designs(), rank=0, world=1, solver=_oracle_solver)
    for r in (0, 1):
        assert np.array_equal(got[r], single)
    assert not np.isnan(single).any()
    assert list(single[:, 0]) == list(range(5))
