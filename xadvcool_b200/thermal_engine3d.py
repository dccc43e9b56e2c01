"""Thermal D3Q19 operators with the names, argument order and semantics of the reference module
src/thermal_engine3d.py, launched as hand-written sm_100a kernels of libxac.so on the current torch
CUDA stream (reference layouts, torch CUDA tensors)."""
from __future__ import annotations

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, dims3, stream_ptr
from .fluid_engine3d import (BC_FLUID, BC_INLET, BC_OUTLET, BC_SOLID, E_CONST, OPPOSITE_CONST,  # noqa: F401
                             W_CONST, _accumulate, _pop_dims, _scratch, field_stats, launch)

F32, I32 = torch.float32, torch.int32


def compute_thermal_equilibrium_kernel(rho, u, T, g_eq, mask):
    """src/thermal_engine3d.py:7-47 (``rho`` is accepted and unused, as in the reference)."""
    nx, ny, nz = dims3(T, "T")
    _capi.call("xac_thermal_equilibrium", dev_ptr(u, F32, "u", (nx, ny, nz, 3)), dev_ptr(T, F32, "T"),
               dev_ptr(g_eq, F32, "g_eq", (19, nx, ny, nz)), dev_ptr(mask, I32, "mask", (nx, ny, nz)),
               nx, ny, nz, stream_ptr())


def thermal_bgk_collision_kernel(g_old, g_eq, g_new, mask, tau_fluid, tau_solid, heat_source_mask,
                                 heat_source_power):
    """src/thermal_engine3d.py:49-86."""
    nx, ny, nz = _pop_dims(g_old, "g_old")
    sh = (19, nx, ny, nz)
    _capi.call("xac_thermal_bgk_collision", dev_ptr(g_old, F32, "g_old"), dev_ptr(g_eq, F32, "g_eq", sh),
               dev_ptr(g_new, F32, "g_new", sh), dev_ptr(mask, I32, "mask", (nx, ny, nz)), float(tau_fluid),
               float(tau_solid), dev_ptr(heat_source_mask, F32, "heat_source_mask", (nx, ny, nz)),
               float(heat_source_power), nx, ny, nz, stream_ptr())


def fused_thermal_equilibrium_collision_kernel(g_old, u, T, g_new, mask, tau_fluid, tau_solid, heat_source_mask,
                                               heat_source_power):
    """src/thermal_engine3d.py:91-145."""
    nx, ny, nz = _pop_dims(g_old, "g_old")
    _capi.call("xac_fused_thermal_collision", dev_ptr(g_old, F32, "g_old"), dev_ptr(u, F32, "u", (nx, ny, nz, 3)),
               dev_ptr(T, F32, "T", (nx, ny, nz)), dev_ptr(g_new, F32, "g_new", (19, nx, ny, nz)),
               dev_ptr(mask, I32, "mask", (nx, ny, nz)), float(tau_fluid), float(tau_solid),
               dev_ptr(heat_source_mask, F32, "heat_source_mask", (nx, ny, nz)), float(heat_source_power),
               nx, ny, nz, stream_ptr())


def thermal_streaming_kernel(g_post_collision, g_streamed, mask, T_inlet, nx, ny, nz):
    """src/thermal_engine3d.py:147-211."""
    sh = (19, nx, ny, nz)
    _capi.call("xac_thermal_stream", dev_ptr(g_post_collision, F32, "g_post_collision", sh),
               dev_ptr(g_streamed, F32, "g_streamed", sh), dev_ptr(mask, I32, "mask", (nx, ny, nz)),
               float(T_inlet), int(nx), int(ny), int(nz), stream_ptr())


def compute_thermal_macroscopic_kernel(g, T):
    """src/thermal_engine3d.py:214-224."""
    nx, ny, nz = _pop_dims(g, "g")
    _capi.call("xac_thermal_macroscopic", dev_ptr(g, F32, "g"), dev_ptr(T, F32, "T", (nx, ny, nz)),
               nx, ny, nz, stream_ptr())


def compute_thermal_stats_kernel(T, stats, u, domain_mask):
    """src/thermal_engine3d.py:226-243: adds [max_t, sum_t, count, Q_out, Q_out_count] into ``stats``."""
    nx, ny, nz = dims3(T, "T")
    rho = _scratch("rho1", (nx, ny, nz), T.device, 1.0)
    s = field_stats(rho, u, T, domain_mask)
    _accumulate(stats, s[11:16], {0})
