"""Many designs solved together by libxac.so's persistent batched kernel (one cooperative launch advances
every active design; designs retire on convergence or divergence and free their share of the GPU).

    b = Batch([dict(mask=m, heat_source=h, tau_fluid=0.55, u_inlet_val=0.03), ...])
    results = b.run(max_steps=30000, tol_ke=1e-6, tol_T=1e-6)
    rho, u, T = b.lattice(3).fields()

An open batch is a queue: designs join while it runs and leave when they finish (design sweeps, sweep.py).

    b = Batch.open()
    slot = b.admit(dict(mask=m, heat_source=h, tau_fluid=0.55, u_inlet_val=0.03))
    for r in b.advance(1000, max_steps=30000, tol_ke=1e-6, tol_T=1e-6):
        scalars = b.lattice(r["slot"]).scalars(); b.release(r["slot"])
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._tensors import stream_ptr
from .lattice import Lattice

_DEFAULTS = dict(tau_fluid=0.52, heat_power=0.1, t_inlet=25.0, u_inlet_val=0.03, Pr=7.0, k_ratio=628.0,
                 rho_outlet=1.0)


def _desc(d: dict, i, precision: str):
    """ABI descriptor of design dict ``d`` -> (desc, mask, heat_source, params); the arrays must outlive the call
    that reads the descriptor."""
    prm = dict(_DEFAULTS)
    prm.update({k: v for k, v in d.items() if k not in ("mask", "heat_source")})
    mask = np.ascontiguousarray(np.asarray(d["mask"]), dtype=np.int32)
    if mask.ndim != 3:
        raise ValueError(f"design {i}: mask must be 3-D")
    hs = d.get("heat_source")
    if hs is not None:
        hs = np.ascontiguousarray(np.array(hs, dtype=np.float32))
        if hs.shape != mask.shape:
            raise ValueError(f"design {i}: heat_source shape {hs.shape} != domain shape {mask.shape}")
    nx, ny, nz = mask.shape
    desc = _capi.Desc(nx, ny, nz, mask.ctypes.data, hs.ctypes.data if hs is not None else None,
                      float(prm["tau_fluid"]), float(prm["Pr"]), float(prm["k_ratio"]), float(prm["u_inlet_val"]),
                      float(prm["rho_outlet"]), float(prm["t_inlet"]), float(prm["heat_power"]),
                      _capi.PRECISIONS[precision])
    prm["precision"] = precision
    return desc, mask, hs, prm


def footprint(design: dict, precision: str = "fp32") -> int:
    """Device bytes a design takes in a batch (populations, link words, fields, reduction rows). Fluid populations
    are stored for the mask's non-solid cells only, so the mask is read."""
    if precision not in _capi.PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_capi.PRECISIONS)}")
    mask = np.ascontiguousarray(np.asarray(design["mask"]), dtype=np.int32)
    if mask.ndim != 3:
        raise ValueError("mask must be 3-D")
    nx, ny, nz = mask.shape
    d = _capi.Desc(nx, ny, nz, mask.ctypes.data, None, 0.6, 1.0, 1.0, 0.0, 1.0, 0.0, 0.0,
                   _capi.PRECISIONS[precision])
    out = C.c_ulonglong()
    _capi.call("xac_lattice_footprint", C.byref(d), C.byref(out))
    return int(out.value)


def _run_opts(max_steps, stats_every, tol_ke, tol_T, min_steps, pump_mode, target_power):
    if pump_mode not in ("constant_flow", "constant_power"):
        raise ValueError(f"unknown pump_mode {pump_mode!r}")
    return _capi.RunOpts(int(max_steps), int(stats_every), float(tol_ke), float(tol_T),
                         1 if pump_mode == "constant_power" else 0, float(target_power), int(min_steps))


def _result(r) -> dict:
    return {"steps": int(r.steps), "converged": bool(r.converged), "diverged": bool(r.diverged), "d_ke": r.d_ke,
            "dT_conv": r.dT_conv, "dQ_conv": r.dQ_conv, "u_inlet_final": r.u_inlet_final,
            "last_stats": np.array(r.last_stats[:], dtype=np.float64)}


class Batch:
    def __init__(self, designs, *, precision="fp32", device="cuda"):
        if not designs:
            raise ValueError("a batch needs at least one design")
        if precision not in _capi.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_capi.PRECISIONS)}")
        self.device = torch.device(device)
        self.precision = precision
        descs = (_capi.Desc * len(designs))()
        keep = []
        self._specs = {}
        for i, d in enumerate(designs):
            descs[i], mask, hs, prm = _desc(d, i, precision)
            keep += [mask, hs]
            self._specs[i] = (mask, prm)
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            _capi.call("xac_batch_create", descs, len(designs), C.byref(self._h), stream_ptr(self.device))
        self.n = len(designs)

    @classmethod
    def open(cls, *, precision="fp32", device="cuda") -> "Batch":
        """An empty batch that designs join (admit) and leave (release) while it runs."""
        if precision not in _capi.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_capi.PRECISIONS)}")
        self = cls.__new__(cls)
        self.device = torch.device(device)
        self.precision = precision
        self._specs = {}
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            _capi.call("xac_batch_open", _capi.PRECISIONS[precision], C.byref(self._h))
        self.n = 0
        return self

    def admit(self, design: dict) -> int:
        """Create ``design`` in a free slot; it joins the running batch at the next stats boundary, from step 0."""
        desc, mask, hs, prm = _desc(design, "admitted", self.precision)
        slot = C.c_int()
        with torch.cuda.device(self.device):
            _capi.call("xac_batch_admit", self._h, C.byref(desc), C.byref(slot), stream_ptr(self.device))
        self._specs[slot.value] = (mask, prm)
        self.n = max(self.n, slot.value + 1)
        return slot.value

    def advance(self, steps: int, max_steps=30000, stats_every=100, tol_ke=1e-7, tol_T=1e-7, min_steps=0,
                pump_mode="constant_flow", target_power=1.0) -> list:
        """Run the open batch for up to ``steps`` steps, returning early after a launch in which designs finished;
        returns those designs, each a result dict (as run() gives) plus "slot" and "gpu_seconds" (its share of the
        launches' wall time)."""
        o = _run_opts(max_steps, stats_every, tol_ke, tol_T, min_steps, pump_mode, target_power)
        cap = C.c_int()
        _capi.call("xac_batch_size", self._h, C.byref(cap))
        n = max(cap.value, 1)
        done, slots = C.c_int(), (C.c_int * n)()
        res, secs = (_capi.RunResult * n)(), (C.c_double * n)()
        with torch.cuda.device(self.device):
            _capi.call("xac_batch_advance", self._h, C.byref(o), int(steps), C.byref(done), slots, res, secs,
                       stream_ptr(self.device))
        out = []
        for k in range(done.value):
            r = _result(res[k])
            r.update(slot=int(slots[k]), gpu_seconds=float(secs[k]))
            out.append(r)
        return out

    def release(self, slot: int):
        """Free a finished design's slot and device memory."""
        _capi.call("xac_batch_release", self._h, int(slot))
        self._specs.pop(slot, None)

    def launch_counts(self):
        """(persistent launches replayed from a captured CUDA graph, direct launches) so far."""
        g, d = C.c_longlong(), C.c_longlong()
        _capi.call("xac_batch_launch_counts", self._h, C.byref(g), C.byref(d))
        return int(g.value), int(d.value)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _capi.load().xac_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return self.n

    def lattice(self, i: int) -> Lattice:
        """Design i as a (borrowed) Lattice: init_fields before run(), fields()/scalars()/stats() after."""
        h = C.c_void_p()
        _capi.call("xac_batch_lattice", self._h, int(i), C.byref(h))
        mask, prm = self._specs[i]
        return Lattice._borrowed(h.value, mask, prm, self.device)

    def tune(self, block: int, steps_per_launch: int):
        _capi.call("xac_batch_tune", self._h, int(block), int(steps_per_launch))

    def get_tune(self):
        b, s = C.c_int(), C.c_int()
        _capi.call("xac_batch_get_tune", self._h, C.byref(b), C.byref(s))
        return int(b.value), int(s.value)

    def run(self, max_steps=30000, stats_every=100, tol_ke=1e-7, tol_T=1e-7, min_steps=0, pump_mode="constant_flow",
            target_power=1.0) -> list:
        """``min_steps`` > 0 replaces the reference's minimum run length (warm-started designs); ``pump_mode``
        "constant_power" runs the reference's pump controller (src/simulation.py:139-146) on every design."""
        o = _run_opts(max_steps, stats_every, tol_ke, tol_T, min_steps, pump_mode, target_power)
        res = (_capi.RunResult * self.n)()
        with torch.cuda.device(self.device):
            _capi.call("xac_batch_run", self._h, C.byref(o), res, stream_ptr(self.device))
        return [_result(r) for r in res]
