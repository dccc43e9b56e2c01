"""ORACLE — test infrastructure only. Numpy restatement of generate_dataset.py:57-179
(compute_hydraulic_diameter, compute_porosity, compute_macroscopic_metrics) used to check the FP64
device reductions of libxac.so. Pinned against the reference function's own outputs in
tests/golden/metrics.json."""
from __future__ import annotations

import numpy as np

BC_SOLID, BC_INLET, BC_OUTLET = 1, 2, 3
BUF, CORE_NX, CORE_NY = 10, 128, 128


def hydraulic_diameter(mask):
    core = mask[BUF:-BUF, 1:-1, 4:-2]
    fl, so = core != BC_SOLID, core == BC_SOLID
    V = int(fl.sum())
    A = int((fl[1:] & so[:-1]).sum() + (so[1:] & fl[:-1]).sum() + (fl[:, 1:] & so[:, :-1]).sum()
            + (so[:, 1:] & fl[:, :-1]).sum() + (fl[:, :, 1:] & so[:, :, :-1]).sum()
            + (so[:, :, 1:] & fl[:, :, :-1]).sum())
    return (4.0 * V / A if A > 0 else float(mask.shape[1])), V, A


def porosity(mask):
    core = mask[BUF:-BUF]
    return 1.0 - np.sum(core == BC_SOLID) / core.size


def macroscopic_metrics(rho, u, T, mask, tau_fluid, u_inlet_val, Dh, A_wetted, Pr=7.0, t_inlet=25.0):
    """generate_dataset.py:80-179, accumulated in float64."""
    rho, u, T = (np.asarray(a, dtype=np.float64) for a in (rho, u, T))
    nx = mask.shape[0]
    outlet_bc = mask[-1] == BC_OUTLET
    in_f, out_f = mask[1] != BC_SOLID, mask[-2] != BC_SOLID
    Q_vol = float(np.sum(u[-1, :, :, 0][outlet_bc]))
    rin = float(np.mean(rho[1][in_f])) if in_f.any() else 1.0
    rout = float(np.mean(rho[-2][out_f])) if out_f.any() else 1.0
    dP = (rin - rout) / 3.0
    P_pump = abs(dP * Q_vol)
    Ts = T[BUF:BUF + CORE_NX, :CORE_NY, 0]
    Tmax, Tavg, Tmin = float(Ts.max()), float(Ts.mean()), float(Ts.min())
    ux_out, T_out = u[-1, :, :, 0][outlet_bc], T[-1][outlet_bc]
    flux = float(ux_out.sum())
    Q_out = float((ux_out * T_out).sum())
    T_out_avg = Q_out / flux if abs(flux) > 1e-12 else t_inlet
    dq = Q_out - t_inlet * flux
    Q_abs = abs(dq) if abs(dq) > 1e-12 else 1e-12
    R_th = (Tmax - t_inlet) / Q_abs
    cf = mask[BUF:-BUF, 1:-1, 4:-2] != BC_SOLID
    T_f = float(T[BUF:-BUF, 1:-1, 4:-2][cf].mean()) if cf.any() else t_inlet
    dT = Tavg - T_f
    h = Q_abs / (A_wetted * abs(dT)) if (abs(dT) > 1e-6 and A_wetted > 0) else 0.0
    k_f = (1.0 / 3.0) * ((0.5 + (tau_fluid - 0.5) / Pr) - 0.5)
    Nu = h * Dh / k_f if k_f > 1e-12 else 0.0
    L = nx - 2 * BUF
    rho_avg = (rin + rout) / 2.0
    f = abs(dP) * Dh / (2.0 * L * rho_avg * u_inlet_val ** 2) if u_inlet_val > 1e-12 else 0.0
    COP = Q_abs / P_pump if P_pump > 1e-12 else 0.0
    return {"R_th": R_th, "Nu": Nu, "f_friction": f, "P_pump": P_pump, "COP": COP, "Q_vol": Q_vol,
            "T_max_surface": Tmax, "T_avg_surface": Tavg, "delta_T_max": Tmax - Tmin,
            "sigma_T": float(Ts.std()), "fluid_temp_rise": T_out_avg - t_inlet, "delta_P": dP}
