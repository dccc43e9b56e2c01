"""Many designs solved together by libxac.so's persistent batched kernel (one cooperative launch advances
every active design; designs retire on convergence or divergence and free their share of the GPU).

    b = Batch([dict(mask=m, heat_source=h, tau_fluid=0.55, u_inlet_val=0.03), ...])
    results = b.run(max_steps=30000, tol_ke=1e-6, tol_T=1e-6)
    rho, u, T = b.lattice(3).fields()
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


class Batch:
    def __init__(self, designs, *, precision="fp32", device="cuda"):
        if not designs:
            raise ValueError("a batch needs at least one design")
        if precision not in _capi.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_capi.PRECISIONS)}")
        self.device = torch.device(device)
        descs = (_capi.Desc * len(designs))()
        self._keep = []
        self._specs = []
        for i, d in enumerate(designs):
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
            self._keep += [mask, hs]
            nx, ny, nz = mask.shape
            descs[i] = _capi.Desc(nx, ny, nz, mask.ctypes.data, hs.ctypes.data if hs is not None else None,
                                  float(prm["tau_fluid"]), float(prm["Pr"]), float(prm["k_ratio"]),
                                  float(prm["u_inlet_val"]), float(prm["rho_outlet"]), float(prm["t_inlet"]),
                                  float(prm["heat_power"]), _capi.PRECISIONS[precision])
            prm["precision"] = precision
            self._specs.append((mask, prm))
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            _capi.call("xac_batch_create", descs, len(designs), C.byref(self._h), stream_ptr(self.device))
        self._keep = []
        self.n = len(designs)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _capi.load().xac_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

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
        if pump_mode not in ("constant_flow", "constant_power"):
            raise ValueError(f"unknown pump_mode {pump_mode!r}")
        o = _capi.RunOpts(int(max_steps), int(stats_every), float(tol_ke), float(tol_T),
                          1 if pump_mode == "constant_power" else 0, float(target_power), int(min_steps))
        res = (_capi.RunResult * self.n)()
        with torch.cuda.device(self.device):
            _capi.call("xac_batch_run", self._h, C.byref(o), res, stream_ptr(self.device))
        return [{"steps": int(r.steps), "converged": bool(r.converged), "diverged": bool(r.diverged),
                 "d_ke": r.d_ke, "dT_conv": r.dT_conv, "dQ_conv": r.dQ_conv, "u_inlet_final": r.u_inlet_final,
                 "last_stats": np.array(r.last_stats[:], dtype=np.float64)} for r in res]
