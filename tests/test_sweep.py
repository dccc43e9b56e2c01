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


def test_footprint_counts_fluid_populations_of_non_solid_cells_only():
    """The queue's memory budget uses the library's footprint: fluid populations (two buffers, 19 per cell) are
    stored for the mask's non-solid cells, in slots rounded up to 32, so a solid cell costs 2 x 19 population
    bytes less than a fluid one. No GPU is needed: the figure is host arithmetic."""
    from xadvcool_b200.batch import footprint
    shape = (10, 6, 5)  # 300 cells: 320 slots all fluid, 32 (the minimum) all solid
    fluid = dict(mask=np.zeros(shape, np.int32))
    solid = dict(mask=np.ones(shape, np.int32))
    for precision, pop_bytes in (("fp32", 4), ("fp16", 2), ("bf16", 2), ("fp32_t16", 4)):
        diff = footprint(fluid, precision) - footprint(solid, precision)
        assert diff == 2 * 19 * pop_bytes * (320 - 32), precision
    half = np.zeros(shape, np.int32)
    half[:, :3, :] = 1  # 150 solid cells: 150 non-solid, 160 slots
    assert footprint(fluid) - footprint(dict(mask=half)) == 2 * 19 * 4 * (320 - 160)


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
                     float(np.abs(r["u"]).max()), 0, 0, 0, 0, 0, 0])
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


class FakeQueue:
    """schedule()'s backend with the open batch's rules and no GPU: admitted designs join at the next multiple of
    stats_every of the batch's step count, each finishes after design["finish"] of its own steps (or max_steps),
    and advance() returns after the stats interval in which designs finished. Scalars are functions of the
    design, GPU seconds its steps x cells."""

    def __init__(self):
        self.step = 0
        self.slots = {}  # slot -> [design, start or None (waiting), done]
        self.max_live = 0
        self.admitted = 0

    def footprint(self, d):
        return int(np.asarray(d["mask"]).size)

    def admit(self, d):
        k = 0
        while k in self.slots:
            k += 1
        self.slots[k] = [d, None, False]
        self.admitted += 1
        self.max_live = max(self.max_live, len(self.slots))
        return k

    def advance(self, steps, max_steps, stats_every, **_):
        out = []
        left = steps
        while left > 0 and not out:
            for v in self.slots.values():
                if v[1] is None and self.step % stats_every == 0:
                    v[1] = self.step
            if not any(v[1] is not None and not v[2] for v in self.slots.values()):
                if not any(v[1] is None for v in self.slots.values()):
                    break
                self.step += stats_every - self.step % stats_every
                continue
            n = min(left, stats_every - self.step % stats_every)
            self.step += n
            left -= n
            for k, v in self.slots.items():
                d, start, done = v
                if start is None or done:
                    continue
                own = self.step - start
                if own >= min(d["finish"], max_steps):
                    v[2] = True
                    out.append({"slot": k, "steps": min(d["finish"], max_steps), "converged": d["finish"] <= max_steps,
                                "diverged": False, "gpu_seconds": own * d["mask"].size * 1e-9})
        return out

    def scalars(self, k):
        d = self.slots[k][0]
        m = np.asarray(d["mask"])
        return {"delta_P": float(d["tau_fluid"]), "R_th": float(m.mean()), "Nu": float(m.shape[0]),
                "pressure_drop": 0.0, "Q_vol": 0.0, "T_max_surface": 0.0, "max_velocity": float(d["u_inlet_val"])}

    def release(self, k):
        assert self.slots[k][2]
        del self.slots[k]


def _queue_designs(n=11):
    rng = np.random.default_rng(4)
    out = []
    for k in range(n):
        m = (rng.random((10 + 2 * (k % 4), 6, 5)) < 0.2).astype(np.int32)
        out.append(dict(mask=m, tau_fluid=0.55 + 0.01 * k, u_inlet_val=0.02 + 0.001 * k, finish=int(rng.integers(2, 40)) * 100 - 37 * (k % 2)))
    return out


def _queue_solver(designs, indices, **kw):
    budget = 3 * 16 * 6 * 5  # at most three of the largest designs at once
    return sweep.schedule(designs, indices, FakeQueue(), budget_bytes=budget, chunk=1000,
                          run=dict(max_steps=3000, stats_every=100))


def test_queue_admits_within_budget_and_refills():
    ds = _queue_designs()
    q = FakeQueue()
    rows = sweep.schedule(ds, list(range(len(ds))), q, budget_bytes=3 * 16 * 6 * 5, chunk=1000,
                          run=dict(max_steps=3000, stats_every=100))
    assert sorted(rows[:, 0]) == list(range(len(ds))) and q.admitted == len(ds)
    assert 2 <= q.max_live <= 4 < len(ds)  # several waves through a batch of at most a few designs
    for r in rows:
        d = ds[int(r[0])]
        assert r[1] == min(d["finish"], 3000) and r[2] == (d["finish"] <= 3000)
        assert r[4] == d["tau_fluid"] and r[10] == d["u_inlet_val"]
    one = sweep.schedule(ds, list(range(len(ds))), FakeQueue(), budget_bytes=10 ** 9, chunk=1000,
                         run=dict(max_steps=3000, stats_every=100))
    key = lambda t: t[np.argsort(t[:, 0])][:, :11]
    assert np.array_equal(key(rows), key(one))  # the budget changes the schedule, not the results


def test_queue_runs_a_design_larger_than_the_budget_alone():
    ds = _queue_designs(3)
    q = FakeQueue()
    rows = sweep.schedule(ds, [0, 1, 2], q, budget_bytes=1, chunk=500, run=dict(max_steps=3000, stats_every=100))
    assert sorted(rows[:, 0]) == [0, 1, 2] and q.max_live == 1


def _queue_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, sweep.run_sweep(_queue_designs(), rank=rank, world=world, solver=_queue_solver)))
    finally:
        dist.destroy_process_group()


def test_two_rank_queue_sweep_with_shards_larger_than_a_batch():
    """Each rank's shard (5-6 designs) runs as several admission waves through a batch that holds at most three;
    the gathered table equals the single-rank one (timing columns aside)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_queue_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    single = sweep.run_sweep(_queue_designs(), rank=0, world=1, solver=_queue_solver)
    for r in (0, 1):
        assert np.array_equal(got[r][:, :11], single[:, :11])
    assert list(single[:, 0]) == list(range(len(_queue_designs())))
