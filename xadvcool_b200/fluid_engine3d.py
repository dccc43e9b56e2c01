"""Fluid D3Q19 operators with the names, argument order and semantics of the reference module
src/fluid_engine3d.py. Each ``*_kernel`` function launches the matching hand-written sm_100a kernel of
libxac.so on the current torch CUDA stream; arrays are torch CUDA tensors in the reference layout
(scalar fields (nx, ny, nz), velocity (nx, ny, nz, 3), populations (19, nx, ny, nz), mask int32).

``launch(kernel, dim, inputs)`` accepts the same call shape as ``wp.launch`` so the reference's
drivers and tests port by replacing the launcher.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi
from ._tensors import dev_ptr, dims3, stream_ptr

# src/fluid_engine3d.py:11-14
BC_FLUID, BC_SOLID, BC_INLET, BC_OUTLET = 0, 1, 2, 3

# src/fluid_engine3d.py:19-39 (rest, 6 faces, 12 edges)
E_CONST = np.array(
    [[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
     [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1],
     [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1]], dtype=np.int32)
# src/fluid_engine3d.py:42-47
W_CONST = np.array([1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12, dtype=np.float64).astype(np.float32)
# src/fluid_engine3d.py:51-53
OPPOSITE_CONST = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17], dtype=np.int32)

F32, I32 = torch.float32, torch.int32


def _pop_dims(f: torch.Tensor, name: str):
    if f.dim() != 4 or f.shape[0] != 19:
        raise ValueError(f"{name}: expected (19, nx, ny, nz), got {tuple(f.shape)}")
    return tuple(int(s) for s in f.shape[1:])


def compute_equilibrium_kernel(rho, u, f_eq):
    """src/fluid_engine3d.py:58-80."""
    nx, ny, nz = dims3(rho, "rho")
    _capi.call("xac_equilibrium", dev_ptr(rho, F32, "rho"), dev_ptr(u, F32, "u", (nx, ny, nz, 3)),
               dev_ptr(f_eq, F32, "f_eq", (19, nx, ny, nz)), nx, ny, nz, stream_ptr())


def compute_macroscopic_kernel(f, rho, u):
    """src/fluid_engine3d.py:85-113."""
    nx, ny, nz = _pop_dims(f, "f")
    _capi.call("xac_macroscopic", dev_ptr(f, F32, "f"), dev_ptr(rho, F32, "rho", (nx, ny, nz)),
               dev_ptr(u, F32, "u", (nx, ny, nz, 3)), nx, ny, nz, stream_ptr())


def bgk_collision_kernel(f_old, f_eq, f_post_collision, domain_mask, tau):
    """src/fluid_engine3d.py:118-136."""
    nx, ny, nz = _pop_dims(f_old, "f_old")
    sh = (19, nx, ny, nz)
    _capi.call("xac_bgk_collision", dev_ptr(f_old, F32, "f_old"), dev_ptr(f_eq, F32, "f_eq", sh),
               dev_ptr(f_post_collision, F32, "f_post_collision", sh),
               dev_ptr(domain_mask, I32, "domain_mask", (nx, ny, nz)), float(tau), nx, ny, nz, stream_ptr())


def fused_equilibrium_collision_kernel(f_old, rho, u, f_post_collision, domain_mask, tau):
    """src/fluid_engine3d.py:141-176."""
    nx, ny, nz = _pop_dims(f_old, "f_old")
    _capi.call("xac_fused_collision", dev_ptr(f_old, F32, "f_old"), dev_ptr(rho, F32, "rho", (nx, ny, nz)),
               dev_ptr(u, F32, "u", (nx, ny, nz, 3)),
               dev_ptr(f_post_collision, F32, "f_post_collision", (19, nx, ny, nz)),
               dev_ptr(domain_mask, I32, "domain_mask", (nx, ny, nz)), float(tau), nx, ny, nz, stream_ptr())


def streaming_kernel(f_post_collision, f_streamed, domain_mask, u_inlet, rho_outlet, nx, ny, nz):
    """src/fluid_engine3d.py:181-272. ``u_inlet`` is a one-element float32 CUDA tensor, read on the device."""
    sh = (19, nx, ny, nz)
    _capi.call("xac_stream", dev_ptr(f_post_collision, F32, "f_post_collision", sh),
               dev_ptr(f_streamed, F32, "f_streamed", sh), dev_ptr(domain_mask, I32, "domain_mask", (nx, ny, nz)),
               dev_ptr(u_inlet, F32, "u_inlet", (1,)), float(rho_outlet), int(nx), int(ny), int(nz), stream_ptr())


_dummy = {}


def _scratch(kind, shape, device, fill):
    key = (kind, shape, str(device))
    t = _dummy.get(key)
    if t is None:
        t = torch.full(shape, fill, dtype=F32, device=device)
        _dummy[key] = t
    return t


def field_stats(rho, u, T, domain_mask):
    """All 17 deterministic FP64 stats (XAC_ST_* order) of the given fields."""
    nx, ny, nz = dims3(rho, "rho")
    out = np.zeros(_capi.NSTATS, dtype=np.float64)
    _capi.call("xac_stats_fields", dev_ptr(rho, F32, "rho"), dev_ptr(u, F32, "u", (nx, ny, nz, 3)),
               dev_ptr(T, F32, "T", (nx, ny, nz)), dev_ptr(domain_mask, I32, "domain_mask", (nx, ny, nz)),
               nx, ny, nz, out.ctypes.data, stream_ptr())
    return out


def _accumulate(stats: torch.Tensor, vals, max_slots):
    cur = stats.detach().to("cpu", torch.float64).numpy()
    for k, v in enumerate(vals):
        cur[k] = max(cur[k], v) if k in max_slots else cur[k] + v
    stats.copy_(torch.from_numpy(cur).to(stats.dtype))


def compute_stats_kernel(rho, u, domain_mask, stats, nx, ny, nz):
    """src/fluid_engine3d.py:277-312: adds the 11 fluid stats into ``stats`` (max into slot 0), like the
    reference's atomics into a zeroed buffer; the sums are formed in FP64 in a fixed order."""
    T = _scratch("T0", (nx, ny, nz), rho.device, 0.0)
    s = field_stats(rho, u, T, domain_mask)
    _accumulate(stats, s[:11], {0})


def launch(kernel, dim=None, inputs=(), device=None, **_):
    """``wp.launch`` call shape: launches ``kernel(*inputs)`` (``dim`` is implied by the arrays)."""
    return kernel(*inputs)
