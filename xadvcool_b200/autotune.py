"""Autotuners for the launch shape of the fused coupled step (threads per block x visiting order) and for the
tile of the persistent batched kernel.

The shape changes only the schedule, never a result (every cell runs the same arithmetic). Candidates are
timed with CUDA events on a scratch lattice built from the same inputs, so the caller's lattice does not
advance. The winner is cached per (device, library build, lattice shape, precision, solid fraction) in a JSON
file (``$XAC_AUTOTUNE_CACHE``, default ``~/.cache/xadvcool_b200/autotune.json``). The library build is a hash of
libxac.so, so shapes timed on other kernels (an older build, another layout) are never reused.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np
import torch

BLOCKS = (64, 128, 256)
VARIANTS = (0, 1)  # 0: one thread per row position; 1: thermal rows staged in shared memory (block = row)


def _cache_path() -> Path:
    return Path(os.environ.get("XAC_AUTOTUNE_CACHE", Path.home() / ".cache" / "xadvcool_b200" / "autotune.json"))


_LIB_ID = None


def _lib_id() -> str:
    """Short hash of the loaded library file (computed once per process)."""
    global _LIB_ID
    if _LIB_ID is None:
        import hashlib
        from . import _capi
        h = hashlib.sha256()
        with open(_capi.LIB_PATH, "rb") as f:
            for chunk in iter(lambda: f.read(1 << 20), b""):
                h.update(chunk)
        _LIB_ID = h.hexdigest()[:12]
    return _LIB_ID


def _key(device, shape, precision, solid_frac) -> str:
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    return f"{name}|lib{_lib_id()}|{shape[0]}x{shape[1]}x{shape[2]}|{precision}|solid{round(solid_frac, 1):.1f}"


def _load_cache() -> dict:
    p = _cache_path()
    try:
        return json.loads(p.read_text())
    except Exception:
        return {}


def _store_cache(c: dict) -> None:
    p = _cache_path()
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(".tmp")
        tmp.write_text(json.dumps(c, indent=1, sort_keys=True))
        tmp.replace(p)
    except OSError:
        pass


def time_config(lat, block: int, variant: int, steps: int = 100, repeats: int = 3) -> float:
    """Mean microseconds per coupled step of ``lat`` with the given launch shape (advances ``lat``)."""
    lat.tune(block, variant)
    lat.step(steps)  # warm-up and graph instantiation
    stream = torch.cuda.current_stream(lat.device)
    best = float("inf")
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        lat.step(steps)
        b.record(stream)
        b.synchronize()
        best = min(best, a.elapsed_time(b) * 1e3 / steps)
    return best


def autotune(mask, *, heat_source=None, precision="fp32", device="cuda", steps=100, use_cache=True,
             lattice_kwargs=None) -> dict:
    """Pick the fastest (block, variant) for this design; returns {"block", "variant", "us_per_step", "table"}."""
    from .lattice import Lattice
    mask = np.asarray(mask)
    dev = torch.device(device)
    key = _key(dev, mask.shape, precision, float((mask == 1).mean()))
    cache = _load_cache() if use_cache else {}
    if key in cache:
        return cache[key]
    kw = dict(lattice_kwargs or {})
    if heat_source is not None or "heat_source" not in kw:
        kw["heat_source"] = heat_source
    table = {}
    with Lattice(mask, precision=precision, device=dev, **kw) as scratch:
        scratch.step(2)
        for v in VARIANTS:
            for b in (BLOCKS if v == 0 else BLOCKS[:1]):  # variant 1 launches one block per row: no block size
                table[f"{b}x{v}"] = round(time_config(scratch, b, v, steps=steps), 3)
    best = min(table, key=table.get)
    b, v = (int(t) for t in best.split("x"))
    res = {"block": b, "variant": v, "us_per_step": table[best], "table": table}
    if use_cache:
        cache[key] = res
        _store_cache(cache)
    return res


BATCH_BLOCKS = (64, 128, 256)


def _time_batch(designs, precision, dev, block, steps, stream) -> float:
    """Microseconds per step of a fresh batch of ``designs`` run ``steps`` steps with tile ``block`` (a batch
    runs once, from step 0)."""
    from .batch import Batch
    b = Batch(designs, precision=precision, device=dev)
    try:
        _, spl = b.get_tune()
        b.tune(block, spl)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        b.run(max_steps=steps, stats_every=100, tol_ke=0.0, tol_T=0.0)
        t1.record(stream)
        t1.synchronize()
        return round(t0.elapsed_time(t1) * 1e3 / steps, 3)
    finally:
        b.close()


def autotune_batch(designs, *, precision="fp32", device="cuda", steps=300, use_cache=True) -> dict:
    """Fastest tile of the persistent batched kernel (threads per block = row positions per tile) for this set of
    designs: each candidate runs ``steps`` steps (stats every 100, no retirement) on a scratch batch built from
    the same designs, timed with CUDA events from the launch to the end of the run; the caller's batch does not
    advance. Cached per (device, number of designs, total cells, precision, solid fraction). Returns {"block",
    "us_per_step", "table"}."""
    dev = torch.device(device)
    cells = sum(int(np.asarray(d["mask"]).size) for d in designs)
    solid = sum(int((np.asarray(d["mask"]) == 1).sum()) for d in designs) / max(cells, 1)
    name = torch.cuda.get_device_name(dev).replace(" ", "_")
    key = f"batch|{name}|lib{_lib_id()}|{len(designs)}|{cells}|{precision}|solid{round(solid, 2):.2f}"
    cache = _load_cache() if use_cache else {}
    if key in cache:
        return cache[key]
    stream = torch.cuda.current_stream(dev)
    _time_batch(designs, precision, dev, BATCH_BLOCKS[-1], steps, stream)  # warm-up (module load, first launch)
    table = {str(b): _time_batch(designs, precision, dev, b, steps, stream) for b in BATCH_BLOCKS}
    best = min(table, key=table.get)
    res = {"block": int(best), "us_per_step": table[best], "table": table}
    if use_cache:
        cache[key] = res
        _store_cache(cache)
    return res


def apply_batch(batch, designs, **kw) -> dict:
    """Autotune the tile for ``designs`` and set it on ``batch`` (built from the same designs)."""
    res = autotune_batch(designs, device=batch.device, **kw)
    _, spl = batch.get_tune()
    batch.tune(res["block"], spl)
    return res


def apply(lat, mask=None, **kw) -> dict:
    """Autotune for ``lat``'s design and set the winning shape on it."""
    res = autotune(lat.mask if mask is None else mask, precision=lat.params["precision"], device=lat.device, **kw)
    lat.tune(res["block"], res["variant"])
    return res
