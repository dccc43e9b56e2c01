"""Design sweeps over one or many GPUs: the dataset-generation loop of generate_dataset.py:365-436 run as
independent shards, one process per GPU.

Designs are independent, so there is no collective on the solve path: each rank takes a disjoint shard of the
design list (balanced by lattice cells, longest first), solves it with the batched persistent kernel, and the
per-design scalar rows are gathered once at the end into one [n_designs, n_cols] FP64 table
(torch.distributed all_gather over NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np
import torch

RESULT_COLS = ["design", "steps", "converged", "diverged", "delta_P", "R_th", "Nu", "pressure_drop", "Q_vol",
               "T_max_surface", "max_velocity", "seconds"]


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


def solve_shard(designs: Sequence[dict], indices: Sequence[int], *, max_steps=30000, tol=1e-5, precision="fp32",
                device="cuda", buf=10, core=(128, 128)) -> np.ndarray:
    """Solve designs[indices] together in one batch on ``device``; one result row per design."""
    import time
    from .batch import Batch
    if not indices:
        return np.zeros((0, len(RESULT_COLS)))
    t0 = time.perf_counter()
    b = Batch([designs[i] for i in indices], precision=precision, device=device)
    res = b.run(max_steps=max_steps, stats_every=100, tol_ke=tol, tol_T=tol)
    rows = []
    for k, i in enumerate(indices):
        sc = b.lattice(k).scalars(buf=buf, core_nx=core[0], core_ny=core[1])
        rows.append([i, res[k]["steps"], res[k]["converged"], res[k]["diverged"], sc["delta_P"], sc["R_th"],
                     sc["Nu"], sc["pressure_drop"], sc["Q_vol"], sc["T_max_surface"], sc["max_velocity"], 0.0])
    dt = time.perf_counter() - t0
    for r in rows:
        r[-1] = dt / len(rows)
    b.close()
    return np.asarray(rows, dtype=np.float64)


def run_sweep(designs: Sequence[dict], *, rank=0, world=1, group=None,
              solver: Callable[..., np.ndarray] = solve_shard, **kw) -> np.ndarray:
    """Shard ``designs`` over ``world`` ranks, solve this rank's shard, gather the full result table."""
    parts = shard([np.asarray(d["mask"]).size for d in designs], world)
    rows = solver(designs, parts[rank], **kw)
    return gather_rows(rows, len(designs), group=group)
