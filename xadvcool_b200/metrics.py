"""Scalar outputs of generate_dataset.py:57-179 (Dh, porosity, delta_P, R_th, Nu, ...), reduced on the GPU
in FP64 by libxac.so. Same function names and arguments as the reference."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._tensors import stream_ptr

BC_SOLID = 1
CORE_NX, CORE_NY, CORE_NZ = 128, 128, 32  # src/geometry.py:15
BUF = 10


def compute_hydraulic_diameter(mask):
    """generate_dataset.py:57-68 (host integer counts; identical to the device count in the scalars)."""
    buf = BUF
    core = np.asarray(mask)[buf:-buf, 1:-1, 4:-2]
    fluid = core != BC_SOLID
    solid = core == BC_SOLID
    V_fluid = int(np.sum(fluid))
    fx = np.sum(fluid[1:] & solid[:-1]) + np.sum(solid[1:] & fluid[:-1])
    fy = np.sum(fluid[:, 1:] & solid[:, :-1]) + np.sum(solid[:, 1:] & fluid[:, :-1])
    fz = np.sum(fluid[:, :, 1:] & solid[:, :, :-1]) + np.sum(solid[:, :, 1:] & fluid[:, :, :-1])
    A_wetted = int(fx + fy + fz)
    Dh = 4.0 * V_fluid / A_wetted if A_wetted > 0 else float(np.shape(mask)[1])
    return Dh, V_fluid, A_wetted


def compute_porosity(mask):
    """generate_dataset.py:71-74."""
    core = np.asarray(mask)[BUF:-BUF, :, :]
    return 1.0 - np.sum(core == BC_SOLID) / core.size


def _as_cuda(a, dtype, device):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def device_scalars(rho, u, T, mask, *, tau_fluid, Pr=7.0, u_inlet_val=0.03, t_inlet=25.0, buf=BUF,
                   core_nx=CORE_NX, core_ny=CORE_NY, device="cuda") -> dict:
    """All scalar outputs from fields (numpy or torch, reference layout) via the FP64 device reduction."""
    dev = torch.device(device)
    rho_t, u_t, T_t = (_as_cuda(a, torch.float32, dev) for a in (rho, u, T))
    m_t = _as_cuda(mask, torch.int32, dev)
    nx, ny, nz = m_t.shape
    p = _capi.ScalarParams(int(buf), int(core_nx), int(core_ny), float(t_inlet), float(tau_fluid), float(Pr),
                           float(u_inlet_val))
    out = np.zeros(_capi.NSCALARS, dtype=np.float64)
    with torch.cuda.device(dev):
        _capi.call("xac_scalars_fields", rho_t.data_ptr(), u_t.data_ptr(), T_t.data_ptr(), m_t.data_ptr(),
                   nx, ny, nz, C.byref(p), out.ctypes.data, stream_ptr(dev))
    return dict(zip(_capi.SCALAR_NAMES, out.tolist()))


def compute_macroscopic_metrics(results, mask, params, Dh, A_wetted, Pr=7.0):
    """generate_dataset.py:80-179: same arguments and returned keys; the sums run on the GPU in FP64.
    Nu and f_friction use the caller's Dh and A_wetted, as the reference does."""
    s = device_scalars(results["rho"], results["u"], results["T"], mask, tau_fluid=params["tau_fluid"], Pr=Pr,
                       u_inlet_val=params["u_inlet_val"], t_inlet=25.0)
    Q_abs, dT_conv = s["Q_absorbed"], s["dT_conv"]
    h_avg = Q_abs / (A_wetted * abs(dT_conv)) if (abs(dT_conv) > 1e-6 and A_wetted > 0) else 0.0
    tau_th_fluid = 0.5 + (params["tau_fluid"] - 0.5) / Pr
    k_fluid = (1.0 / 3.0) * (tau_th_fluid - 0.5)
    Nu = (h_avg * Dh / k_fluid) if k_fluid > 1e-12 else 0.0
    nx = np.shape(mask)[0]
    L = nx - 2 * BUF
    u_in = params["u_inlet_val"]
    f = (abs(s["delta_P"]) * Dh) / (2.0 * L * s["rho_avg"] * u_in ** 2) if u_in > 1e-12 else 0.0
    return {
        "R_th": float(s["R_th"]), "Nu": float(Nu), "f_friction": float(f), "P_pump": float(s["P_pump"]),
        "COP": float(s["COP"]), "Q_vol": float(s["Q_vol"]), "T_max_surface": float(s["T_max_surface"]),
        "T_avg_surface": float(s["T_avg_surface"]), "delta_T_max": float(s["delta_T_max"]),
        "sigma_T": float(s["sigma_T"]), "fluid_temp_rise": float(s["fluid_temp_rise"]),
    }
