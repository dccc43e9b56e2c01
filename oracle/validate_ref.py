"""Test infrastructure (not product code): numpy restatement of the reference's physical validators,
analyze_dataset.py:184-323 (validate_sample), on in-memory arrays instead of an HDF5 group. Used only by the
tests, as the checker of xadvcool_b200.validate. Pinned against the reference function itself
(tests/golden/validate.json, made by tests/golden/make_golden.py)."""
from __future__ import annotations

import numpy as np

BC_SOLID, BC_INLET, BC_OUTLET = 1, 2, 3
# analyze_dataset.py:111-120
THRESHOLDS = {
    "mass_conservation": {"pass": 0.01, "warn": 0.05},
    "mach_number": {"pass": 0.15, "warn": 0.30},
    "density_deviation": {"pass": 0.05, "warn": 0.10},
    "temp_lower_bound": {"pass": 0.0, "warn": -0.5},
    "nusselt_low": 1.0,
    "nusselt_high": 500.0,
    "f_re_high": 200.0,
    "divergence_free": {"pass": 0.001, "warn": 0.01},
}


def validate_arrays(mask, u, T, P, hs, attrs, t_inlet=25.0):
    """analyze_dataset.py:184-323 with the group's datasets passed in (P = rho / 3)."""
    fluid = (mask != BC_SOLID)
    c = {}
    rho = P * 3.0                                                          # :200
    inlet_bc = (mask[0, :, :] == BC_INLET)
    outlet_bc = (mask[-1, :, :] == BC_OUTLET)
    inlet_fluid = (mask[1, :, :] != BC_SOLID)
    outlet_fluid = (mask[-2, :, :] != BC_SOLID)
    mdot_in = float(np.sum(rho[1, :, :][inlet_fluid] * u[1, :, :, 0][inlet_fluid]))
    mdot_out = float(np.sum(rho[-2, :, :][outlet_fluid] * u[-2, :, :, 0][outlet_fluid]))
    c["mass_err"] = abs(mdot_in - mdot_out) / (abs(mdot_in) + 1e-12)      # :207
    c["mass_pass"] = c["mass_err"] < THRESHOLDS["mass_conservation"]["pass"]
    c["mass_warn"] = c["mass_err"] < THRESHOLDS["mass_conservation"]["warn"]
    v_mag = np.linalg.norm(u, axis=-1)                                     # :214
    max_v = float(np.max(v_mag[fluid])) if np.any(fluid) else 0.0
    mach = max_v * np.sqrt(3.0)
    c["mach"] = mach
    c["mach_pass"] = mach < THRESHOLDS["mach_number"]["pass"]
    c["mach_warn"] = mach < THRESHOLDS["mach_number"]["warn"]
    rho_dev = float(np.max(np.abs(rho[fluid] - 1.0))) if np.any(fluid) else 0.0   # :222
    c["rho_dev"] = rho_dev
    c["rho_dev_pass"] = rho_dev < max(THRESHOLDS["density_deviation"]["pass"], 2.0 * mach ** 2)
    c["rho_dev_warn"] = rho_dev < max(THRESHOLDS["density_deviation"]["warn"], 3.0 * mach ** 2)
    T_min_fluid = float(np.min(T[fluid])) if np.any(fluid) else t_inlet   # :229
    c["T_lower_bound"] = T_min_fluid - t_inlet
    c["T_lb_pass"] = c["T_lower_bound"] >= THRESHOLDS["temp_lower_bound"]["pass"]
    c["T_lb_warn"] = c["T_lower_bound"] >= THRESHOLDS["temp_lower_bound"]["warn"]
    rho_in = float(np.mean(rho[1, :, :]))                                  # :236
    rho_out = float(np.mean(rho[-2, :, :]))
    c["delta_P"] = (rho_in - rho_out) / 3.0
    c["delta_P_pass"] = c["delta_P"] > 0
    Nu = attrs.get("Nu", 0.0)                                              # :243
    c["Nu"] = Nu
    c["Nu_pass"] = THRESHOLDS["nusselt_low"] <= Nu <= THRESHOLDS["nusselt_high"]
    f_Re = attrs.get("f_friction", 0.0) * attrs.get("Re", 1.0)             # :249
    c["f_Re"] = f_Re
    c["f_Re_pass"] = 0 < f_Re < THRESHOLDS["f_re_high"]
    ux, uy, uz = u[:, :, :, 0], u[:, :, :, 1], u[:, :, :, 2]               # :256
    div_u = ((ux[2:, 1:-1, 1:-1] - ux[:-2, 1:-1, 1:-1]) / 2.0 + (uy[1:-1, 2:, 1:-1] - uy[1:-1, :-2, 1:-1]) / 2.0
             + (uz[1:-1, 1:-1, 2:] - uz[1:-1, 1:-1, :-2]) / 2.0)
    interior = fluid[1:-1, 1:-1, 1:-1]
    if np.any(interior):
        c["mean_div"] = float(np.mean(np.abs(div_u[interior])))
        c["max_div"] = float(np.max(np.abs(div_u[interior])))
    else:
        c["mean_div"], c["max_div"] = 0.0, 0.0
    c["div_pass"] = c["mean_div"] < THRESHOLDS["divergence_free"]["pass"]
    c["div_warn"] = c["mean_div"] < THRESHOLDS["divergence_free"]["warn"]
    heat_power = attrs.get("heat_power", 0.0)                              # :272
    Pr = attrs.get("Pr", 7.0)
    k_ratio = attrs.get("k_ratio", 628.0)
    tau_th_fluid = 0.5 + (attrs.get("tau_fluid", 0.52) - 0.5) / Pr
    tau_th_solid = 0.5 + k_ratio * (tau_th_fluid - 0.5)
    Q_source_rate = (1.0 - 0.5 / tau_th_solid) * heat_power * float(np.sum(hs))
    k_fluid = (1.0 / 3.0) * (tau_th_fluid - 0.5)
    k_solid = (1.0 / 3.0) * (tau_th_solid - 0.5)
    k_in = np.where(mask[1, :, :] == BC_SOLID, k_solid, k_fluid)
    k_out = np.where(mask[-2, :, :] == BC_SOLID, k_solid, k_fluid)
    ux_in = u[0, :, :, 0][inlet_bc] if np.any(inlet_bc) else np.array([0.0])
    ux_out = u[-1, :, :, 0][outlet_bc] if np.any(outlet_bc) else np.array([0.0])
    T_out_bc = T[-1, :, :][outlet_bc] if np.any(outlet_bc) else np.array([t_inlet])
    Q_adv_in = t_inlet * float(np.sum(ux_in))
    Q_adv_out = float(np.sum(ux_out * T_out_bc))
    Q_diff_in = float(np.sum(-k_in * (T[1, :, :] - T[0, :, :])))
    Q_diff_out = float(np.sum(-k_out * (T[-1, :, :] - T[-2, :, :])))
    Q_removed = (Q_adv_out + Q_diff_out) - (Q_adv_in + Q_diff_in)
    c["Q_source_rate"] = Q_source_rate
    c["Q_conv"] = Q_removed
    c["energy_err"] = (abs(Q_source_rate - Q_removed) / (abs(Q_source_rate) + 1e-12)
                       if abs(Q_source_rate) > 1e-12 else 0.0)
    c["energy_pass"] = c["energy_err"] < 0.20
    c["energy_warn"] = c["energy_err"] < 0.40
    return c


def raw_sums(mask, rho, u, T, hs, heat_power, tau_fluid=0.55, Pr=7.0, k_ratio=628.0):
    """The XAC_VAL_* reductions of xac_lattice_validate restated in numpy (float32 per-cell terms, float64 sums):
    the inputs of xadvcool_b200.validate.checks_from_raw."""
    fluid = mask != BC_SOLID
    tth_f = 0.5 + (tau_fluid - 0.5) / Pr
    tth_s = 0.5 + k_ratio * (tth_f - 0.5)
    k_f, k_s = (1.0 / 3.0) * (tth_f - 0.5), (1.0 / 3.0) * (tth_s - 0.5)
    r = {}
    f1, f2 = fluid[1], fluid[-2]
    r["mdot_in"] = float(np.sum((rho[1] * u[1, :, :, 0])[f1].astype(np.float64)))
    r["mdot_out"] = float(np.sum((rho[-2] * u[-2, :, :, 0])[f2].astype(np.float64)))
    vm = np.sqrt(u[..., 0] * u[..., 0] + u[..., 1] * u[..., 1] + u[..., 2] * u[..., 2])
    r["max_v"] = float(vm[fluid].max())
    r["rho_dev"] = float(np.abs(rho[fluid] - np.float32(1.0)).max())
    r["T_min"] = float(T[fluid].min())
    r["n_fluid"] = float(fluid.sum())
    r["rho1_all"] = float(rho[1].astype(np.float64).sum())
    r["rho2_all"] = float(rho[-2].astype(np.float64).sum())
    ux, uy, uz = u[..., 0], u[..., 1], u[..., 2]
    d = ((ux[2:, 1:-1, 1:-1] - ux[:-2, 1:-1, 1:-1]) / np.float32(2.0)
         + (uy[1:-1, 2:, 1:-1] - uy[1:-1, :-2, 1:-1]) / np.float32(2.0)) \
        + (uz[1:-1, 1:-1, 2:] - uz[1:-1, 1:-1, :-2]) / np.float32(2.0)
    inner = fluid[1:-1, 1:-1, 1:-1]
    ad = np.abs(d[inner]).astype(np.float64)
    r["div_sum"], r["div_max"], r["div_n"] = float(ad.sum()), float(ad.max()), float(inner.sum())
    r["q_src"] = float(heat_power) * float(np.asarray(hs, np.float64).sum())
    r["adv_in"] = float(u[0, :, :, 0][mask[0] == BC_INLET].astype(np.float64).sum())
    r["adv_out"] = float((u[-1, :, :, 0] * T[-1])[mask[-1] == BC_OUTLET].astype(np.float64).sum())
    k_in = np.where(mask[1] == BC_SOLID, k_s, k_f)
    k_out = np.where(mask[-2] == BC_SOLID, k_s, k_f)
    r["diff_in"] = float(np.sum(-k_in * (T[1] - T[0]).astype(np.float64)))
    r["diff_out"] = float(np.sum(-k_out * (T[-1] - T[-2]).astype(np.float64)))
    return r
