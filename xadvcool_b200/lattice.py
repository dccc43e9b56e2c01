"""Python handle on one fused coupled lattice of libxac.so (the path of src/simulation.py:14-162)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, stream_ptr


def derived_taus(tau_fluid: float, Pr: float, k_ratio: float):
    """src/simulation.py:70-71."""
    tau_th_fluid = 0.5 + ((tau_fluid - 0.5) / Pr)
    tau_th_solid = 0.5 + k_ratio * (tau_th_fluid - 0.5)
    return tau_th_fluid, tau_th_solid


class Lattice:
    """One design: mask + heat source + physical parameters, populations resident on the GPU.

    ``step(n)`` advances n coupled steps, each equal to one replay of the reference's six-kernel graph.
    """

    def __init__(self, mask, *, tau_fluid=0.52, heat_power=0.1, t_inlet=25.0, u_inlet_val=0.03, heat_source=None,
                 Pr=7.0, k_ratio=628.0, rho_outlet=1.0, precision="fp32", device="cuda"):
        mask_np = np.ascontiguousarray(np.asarray(mask), dtype=np.int32)
        if mask_np.ndim != 3:
            raise ValueError(f"mask must be 3-D (nx, ny, nz), got shape {mask_np.shape}")
        nx, ny, nz = mask_np.shape
        hs_np = None
        if heat_source is not None:
            hs_np = np.ascontiguousarray(np.array(heat_source, dtype=np.float32))
            if hs_np.shape != (nx, ny, nz):
                raise ValueError(f"heat_source shape {hs_np.shape} != domain shape ({nx}, {ny}, {nz})")
        if precision not in _capi.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_capi.PRECISIONS)}, got {precision!r}")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the solver runs on CUDA devices only")
        self.shape = (nx, ny, nz)
        self.params = dict(tau_fluid=float(tau_fluid), heat_power=float(heat_power), t_inlet=float(t_inlet),
                           u_inlet_val=float(u_inlet_val), Pr=float(Pr), k_ratio=float(k_ratio),
                           rho_outlet=float(rho_outlet), precision=precision)
        d = _capi.Desc(nx, ny, nz, mask_np.ctypes.data, hs_np.ctypes.data if hs_np is not None else None,
                       float(tau_fluid), float(Pr), float(k_ratio), float(u_inlet_val), float(rho_outlet),
                       float(t_inlet), float(heat_power), _capi.PRECISIONS[precision])
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_create", C.byref(d), C.byref(self._h), stream_ptr(self.device))
        self.mask = mask_np

    @classmethod
    def _borrowed(cls, handle, mask, params, device):
        """A view of a lattice owned by someone else (a batch): never destroyed from here."""
        self = cls.__new__(cls)
        self._h = C.c_void_p(handle)
        self._owner = False
        self.mask = np.ascontiguousarray(mask, dtype=np.int32)
        self.shape = self.mask.shape
        self.params = dict(params)
        self.device = torch.device(device)
        return self

    # -- lifecycle -------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_owner", True) and getattr(self, "_h", None) is not None and self._h.value:
            _capi.load().xac_lattice_destroy(self._h)
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

    # -- stepping --------------------------------------------------------------------------------
    def init_fields(self, rho=None, u=None, T=None):
        """Warm start: populations at the equilibria of the given fields (reference layout, CUDA tensors)."""
        nx, ny, nz = self.shape
        p = [dev_ptr(rho, torch.float32, "rho", (nx, ny, nz)) if rho is not None else None,
             dev_ptr(u, torch.float32, "u", (nx, ny, nz, 3)) if u is not None else None,
             dev_ptr(T, torch.float32, "T", (nx, ny, nz)) if T is not None else None]
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_init_fields", self._h, *p, stream_ptr(self.device))

    def step(self, n: int = 1):
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_step", self._h, int(n), stream_ptr(self.device))

    @property
    def steps_done(self) -> int:
        v = C.c_longlong()
        _capi.call("xac_lattice_steps_done", self._h, C.byref(v))
        return int(v.value)

    def tune(self, block: int, variant: int):
        """Launch shape of the fused step: threads per block (64, 128, 256) and variant (0: one thread per row
        position; 1: one block per row with the thermal input staged in shared memory). Results are unaffected."""
        _capi.call("xac_lattice_tune", self._h, int(block), int(variant))

    def pattern_copy_us(self, launches: int = 200) -> float:
        """Microseconds per launch of a kernel that moves exactly the step's populations with no arithmetic (the
        memory-pattern floor of the step for this design); leaves the lattice at the cold start (step 0)."""
        us = C.c_double()
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_pattern_copy", self._h, int(launches), C.byref(us), stream_ptr(self.device))
        return float(us.value)

    def get_tune(self):
        b, v = C.c_int(), C.c_int()
        _capi.call("xac_lattice_get_tune", self._h, C.byref(b), C.byref(v))
        return int(b.value), int(v.value)

    def set_inlet(self, u_in: float):
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_set_inlet", self._h, float(u_in), stream_ptr(self.device))

    def get_inlet(self) -> float:
        v = C.c_double()
        _capi.call("xac_lattice_get_inlet", self._h, C.byref(v), None)
        return float(v.value)

    # -- observation -----------------------------------------------------------------------------
    def stats(self) -> np.ndarray:
        out = np.zeros(_capi.NSTATS, dtype=np.float64)
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_stats", self._h, out.ctypes.data, stream_ptr(self.device))
        return out

    def fields(self):
        """(rho, u, T) as CUDA tensors in the reference layout."""
        nx, ny, nz = self.shape
        rho = torch.empty((nx, ny, nz), dtype=torch.float32, device=self.device)
        u = torch.empty((nx, ny, nz, 3), dtype=torch.float32, device=self.device)
        T = torch.empty((nx, ny, nz), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_fields", self._h, rho.data_ptr(), u.data_ptr(), T.data_ptr(),
                       stream_ptr(self.device))
        return rho, u, T

    def scalars(self, buf=10, core_nx=128, core_ny=128, t_inlet=25.0, Pr=None, u_inlet=None) -> dict:
        """generate_dataset.py:80-179 on the device in FP64 (plus Dh, A_wetted, porosity, pressure_drop)."""
        p = _capi.ScalarParams(int(buf), int(core_nx), int(core_ny), float(t_inlet), self.params["tau_fluid"],
                               float(self.params["Pr"] if Pr is None else Pr),
                               float(self.params["u_inlet_val"] if u_inlet is None else u_inlet))
        out = np.zeros(_capi.NSCALARS, dtype=np.float64)
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_scalars", self._h, C.byref(p), out.ctypes.data, stream_ptr(self.device))
        return dict(zip(_capi.SCALAR_NAMES, out.tolist()))

    def validate_raw(self) -> dict:
        """FP64 device reductions behind the physical validators (XAC_VAL_* slots by name)."""
        out = np.zeros(_capi.NVALIDATE, dtype=np.float64)
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_validate", self._h, out.ctypes.data, stream_ptr(self.device))
        return dict(zip(_capi.VALIDATE_NAMES, out.tolist()))

    # -- native loop -----------------------------------------------------------------------------
    def run(self, max_steps=40000, stats_every=100, tol_ke=1e-7, tol_T=1e-7, pump_mode="constant_flow",
            target_power=1.0, min_steps=0) -> dict:
        """src/simulation.py:102-162 in native code; returns steps / convergence diagnostics.

        ``min_steps`` > 0 replaces the reference's minimum run length before convergence may be declared
        (min(0.6 max_steps, max(5000, 2 nx / u_in)), src/simulation.py:102-104): warm starts use a short one."""
        if pump_mode not in ("constant_flow", "constant_power"):
            raise ValueError(f"unknown pump_mode {pump_mode!r}")
        o = _capi.RunOpts(int(max_steps), int(stats_every), float(tol_ke), float(tol_T),
                          1 if pump_mode == "constant_power" else 0, float(target_power), int(min_steps))
        r = _capi.RunResult()
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_run", self._h, C.byref(o), C.byref(r), stream_ptr(self.device))
        return {"steps": int(r.steps), "converged": bool(r.converged), "diverged": bool(r.diverged),
                "d_ke": r.d_ke, "dT_conv": r.dT_conv, "dQ_conv": r.dQ_conv, "u_inlet_final": r.u_inlet_final,
                "last_stats": np.array(r.last_stats[:], dtype=np.float64)}

    # -- checkpoint ------------------------------------------------------------------------------
    def state_bytes(self) -> int:
        v = C.c_size_t()
        _capi.call("xac_lattice_state_bytes", self._h, C.byref(v))
        return int(v.value)

    def save_state(self) -> bytes:
        n = self.state_bytes()
        buf = (C.c_char * n)()
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_save_state", self._h, C.addressof(buf), n, stream_ptr(self.device))
        return bytes(buf)

    def load_state(self, blob: bytes):
        n = self.state_bytes()
        if len(blob) < n:
            raise ValueError(f"state blob has {len(blob)} bytes, expected {n}")
        buf = C.create_string_buffer(blob, len(blob))
        with torch.cuda.device(self.device):
            _capi.call("xac_lattice_load_state", self._h, C.addressof(buf), len(blob), stream_ptr(self.device))


def reference_run_fp64(mask, steps: int, *, tau_fluid=0.52, heat_power=0.1, t_inlet=25.0, u_inlet_val=0.03,
                       heat_source=None, Pr=7.0, k_ratio=628.0, rho_outlet=1.0, device="cuda"):
    """FP64 solve on the GPU (the oracle for the reduced-precision storage forms): cold start, then ``steps``
    replays of the reference's six-kernel step (src/simulation.py:60-100) in double precision. Returns (rho, u, T)
    as float64 CUDA tensors in the reference layout."""
    mask_np = np.ascontiguousarray(np.asarray(mask), dtype=np.int32)
    if mask_np.ndim != 3:
        raise ValueError(f"mask must be 3-D (nx, ny, nz), got shape {mask_np.shape}")
    nx, ny, nz = mask_np.shape
    hs_np = None
    if heat_source is not None:
        hs_np = np.ascontiguousarray(np.array(heat_source, dtype=np.float32))
        if hs_np.shape != (nx, ny, nz):
            raise ValueError(f"heat_source shape {hs_np.shape} != domain shape ({nx}, {ny}, {nz})")
    dev = torch.device(device)
    d = _capi.Desc(nx, ny, nz, mask_np.ctypes.data, hs_np.ctypes.data if hs_np is not None else None,
                   float(tau_fluid), float(Pr), float(k_ratio), float(u_inlet_val), float(rho_outlet), float(t_inlet),
                   float(heat_power), _capi.PRECISIONS["fp32"])
    rho = torch.empty((nx, ny, nz), dtype=torch.float64, device=dev)
    u = torch.empty((nx, ny, nz, 3), dtype=torch.float64, device=dev)
    T = torch.empty((nx, ny, nz), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        _capi.call("xac_reference_run_fp64", C.byref(d), int(steps), rho.data_ptr(), u.data_ptr(), T.data_ptr(),
                   stream_ptr(dev))
    return rho, u, T
