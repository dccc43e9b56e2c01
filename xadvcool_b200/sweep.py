"""Design sweeps over one or many GPUs: the dataset-generation loop of generate_dataset.py:365-436 run as
independent shards, one process per GPU.

Designs are independent, so there is no collective on the solve path: each rank takes a disjoint shard of the
design list (balanced by lattice cells, longest first), solves it with the batched persistent kernel, and the
per-design scalar rows are gathered once at the end into one [n_designs, n_cols] FP64 table
(torch.distributed all_gather over NCCL on GPUs, gloo on CPU).

A shard runs as a queue over one open batch (schedule()): designs join while their device footprint fits an HBM
budget and the batch's 1024 slots, and every design that finishes (converged, diverged or at the step limit) is
read out and released, and its slot and memory go to the next design of the queue. Per design the table records
`seconds`, its share of the GPU's wall time (each persistent launch's time split among the designs in it by their
cells), and `latency_s`, the wall time from its admission to the end of the launch it finished in.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np
import torch

RESULT_COLS = ["design", "steps", "converged", "diverged", "delta_P", "R_th", "Nu", "pressure_drop", "Q_vol",
               "T_max_surface", "max_velocity", "seconds", "latency_s"]


def shard(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time assignment of designs (by cost, e.g. cell count) to ``world`` ranks.
    Deterministic: ties are broken by design index. Returns the design indices of every rank, ascending."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def gather_rows(rows: np.ndarray, n_total: int, group=None) -> np.ndarray:
    """Gather every rank's [n_local, n_cols] FP64 rows (first column = global design index) into the full
    [n_total, n_cols] table ordered by design index. Works on any backend (one all_gather of a padded tensor)."""
    import torch.distributed as dist
    rows = np.asarray(rows, dtype=np.float64).reshape(-1, len(RESULT_COLS))
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        table = np.full((n_total, len(RESULT_COLS)), np.nan)
        for r in rows:
            table[int(r[0])] = r
        return table
    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    n_max = torch.tensor([rows.shape[0]], dtype=torch.int64, device=dev)
    dist.all_reduce(n_max, op=dist.ReduceOp.MAX, group=group)
    pad = np.full((int(n_max.item()), len(RESULT_COLS)), -1.0)
    pad[: rows.shape[0]] = rows
    mine = torch.from_numpy(pad).to(dev)
    out = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(out, mine, group=group)
    table = np.full((n_total, len(RESULT_COLS)), np.nan)
    for t in out:
        for r in t.cpu().numpy():
            if r[0] >= 0:
                table[int(r[0])] = r
    return table


class BatchQueue:
    """The GPU side of schedule(): an open batch whose finished designs are read out (scalars) and released."""

    def __init__(self, precision="fp32", device="cuda", buf=10, core=(128, 128), steps_per_launch=None):
        from .batch import Batch
        self.precision, self.buf, self.core = precision, buf, core
        self.batch = Batch.open(precision=precision, device=device)
        if steps_per_launch:
            self.batch.tune(self.batch.get_tune()[0], int(steps_per_launch))

    def footprint(self, design) -> int:
        from .batch import footprint
        return footprint(design, self.precision)

    def admit(self, design) -> int:
        return self.batch.admit(design)

    def advance(self, steps, **run) -> list:
        return self.batch.advance(steps, **run)

    def scalars(self, slot) -> dict:
        return self.batch.lattice(slot).scalars(buf=self.buf, core_nx=self.core[0], core_ny=self.core[1])

    def release(self, slot) -> None:
        self.batch.release(slot)

    def close(self) -> None:
        self.batch.close()


def schedule(designs: Sequence[dict], indices: Sequence[int], backend, *, budget_bytes: int, max_slots: int = 1024,
             chunk: int = 1000, run: dict) -> np.ndarray:
    """Solve designs[indices] through ``backend`` (BatchQueue, or any object with its methods): largest designs
    first, admitted while the footprints of the designs in the batch stay within ``budget_bytes`` and
    ``max_slots`` (one design always runs, whatever its size); each finished design is read out and released and
    the queue refills its slot. ``run``: the convergence options of Batch.advance. One result row per design, in
    the order they finished."""
    import time
    queue = sorted(indices, key=lambda i: (-int(np.asarray(designs[i]["mask"]).size), i))
    live = {}  # slot -> (design index, footprint, admission time)
    used = 0
    rows = []
    while queue or live:
        while queue and len(live) < max_slots:
            need = backend.footprint(designs[queue[0]])
            if live and used + need > budget_bytes:
                break
            i = queue.pop(0)
            live[backend.admit(designs[i])] = (i, need, time.perf_counter())
            used += need
        for f in backend.advance(chunk, **run):
            i, need, t_in = live.pop(f["slot"])
            sc = backend.scalars(f["slot"])
            rows.append([i, f["steps"], f["converged"], f["diverged"], sc["delta_P"], sc["R_th"], sc["Nu"],
                         sc["pressure_drop"], sc["Q_vol"], sc["T_max_surface"], sc["max_velocity"],
                         f["gpu_seconds"], time.perf_counter() - t_in])
            backend.release(f["slot"])
            used -= need
    return np.asarray(rows, dtype=np.float64).reshape(-1, len(RESULT_COLS))


def solve_shard(designs: Sequence[dict], indices: Sequence[int], *, max_steps=30000, tol=1e-5, precision="fp32",
                device="cuda", buf=10, core=(128, 128), budget_bytes=None, max_slots=1024, chunk=1000,
                steps_per_launch=None) -> np.ndarray:
    """Solve designs[indices] on ``device`` as a queue over one open batch (schedule()); ``budget_bytes`` defaults
    to 80% of the device memory free at the start. One result row per design."""
    if not indices:
        return np.zeros((0, len(RESULT_COLS)))
    if budget_bytes is None:
        free, _ = torch.cuda.mem_get_info(torch.device(device))
        budget_bytes = int(0.8 * free)
    q = BatchQueue(precision, device, buf, core, steps_per_launch)
    try:
        return schedule(designs, indices, q, budget_bytes=budget_bytes, max_slots=max_slots, chunk=chunk,
                        run=dict(max_steps=max_steps, stats_every=100, tol_ke=tol, tol_T=tol))
    finally:
        q.close()


def run_sweep(designs: Sequence[dict], *, rank=0, world=1, group=None,
              solver: Callable[..., np.ndarray] = solve_shard, **kw) -> np.ndarray:
    """Shard ``designs`` over ``world`` ranks, solve this rank's shard, gather the full result table."""
    parts = shard([np.asarray(d["mask"]).size for d in designs], world)
    rows = solver(designs, parts[rank], **kw)
    return gather_rows(rows, len(designs), group=group)
