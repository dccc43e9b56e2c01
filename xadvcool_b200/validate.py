"""Physical validators of a solved design (analyze_dataset.py:184-323, the reference's validate_sample), with
every field reduction done on the GPU in FP64 (xac_lattice_validate) and Nu, f and D_h taken from the device
scalars. Thresholds and check names are the reference's.

    checks = validate(lattice)            # {"mass_err": ..., "mass_pass": ..., ..., "energy_err": ...}
"""
from __future__ import annotations

import math

# analyze_dataset.py:111-120 (kept identical: the pass/warn verdicts must mean the same)
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


def checks_from_raw(raw: dict, attrs: dict, plane_cells: int, t_inlet: float = 25.0) -> dict:
    """The reference's checks from the device reductions (``raw``: XAC_VAL_* slots by name, see _capi) and the
    design's attributes (heat_power, Pr, k_ratio, tau_fluid, Nu, f_friction, Re). ``plane_cells`` = ny*nz."""
    T_ = THRESHOLDS
    c = {}
    c["mass_err"] = abs(raw["mdot_in"] - raw["mdot_out"]) / (abs(raw["mdot_in"]) + 1e-12)
    c["mass_pass"] = c["mass_err"] < T_["mass_conservation"]["pass"]
    c["mass_warn"] = c["mass_err"] < T_["mass_conservation"]["warn"]
    has_fluid = raw["n_fluid"] > 0
    mach = (raw["max_v"] if has_fluid else 0.0) * math.sqrt(3.0)
    c["mach"] = mach
    c["mach_pass"] = mach < T_["mach_number"]["pass"]
    c["mach_warn"] = mach < T_["mach_number"]["warn"]
    rho_dev = raw["rho_dev"] if has_fluid else 0.0
    c["rho_dev"] = rho_dev
    c["rho_dev_pass"] = rho_dev < max(T_["density_deviation"]["pass"], 2.0 * mach ** 2)
    c["rho_dev_warn"] = rho_dev < max(T_["density_deviation"]["warn"], 3.0 * mach ** 2)
    c["T_lower_bound"] = (raw["T_min"] if has_fluid else t_inlet) - t_inlet
    c["T_lb_pass"] = c["T_lower_bound"] >= T_["temp_lower_bound"]["pass"]
    c["T_lb_warn"] = c["T_lower_bound"] >= T_["temp_lower_bound"]["warn"]
    c["delta_P"] = (raw["rho1_all"] / plane_cells - raw["rho2_all"] / plane_cells) / 3.0
    c["delta_P_pass"] = c["delta_P"] > 0
    Nu = attrs.get("Nu", 0.0)
    c["Nu"] = Nu
    c["Nu_pass"] = T_["nusselt_low"] <= Nu <= T_["nusselt_high"]
    c["f_Re"] = attrs.get("f_friction", 0.0) * attrs.get("Re", 1.0)
    c["f_Re_pass"] = 0 < c["f_Re"] < T_["f_re_high"]
    if raw["div_n"] > 0:
        c["mean_div"], c["max_div"] = raw["div_sum"] / raw["div_n"], raw["div_max"]
    else:
        c["mean_div"], c["max_div"] = 0.0, 0.0
    c["div_pass"] = c["mean_div"] < T_["divergence_free"]["pass"]
    c["div_warn"] = c["mean_div"] < T_["divergence_free"]["warn"]
    Pr = attrs.get("Pr", 7.0)
    tau_th_fluid = 0.5 + (attrs.get("tau_fluid", 0.52) - 0.5) / Pr
    tau_th_solid = 0.5 + attrs.get("k_ratio", 628.0) * (tau_th_fluid - 0.5)
    # the source is on the z = 0 floor, which is solid (analyze_dataset.py:276-277)
    q_src = (1.0 - 0.5 / tau_th_solid) * raw["q_src"]
    q_removed = (raw["adv_out"] + raw["diff_out"]) - (t_inlet * raw["adv_in"] + raw["diff_in"])
    c["Q_source_rate"] = q_src
    c["Q_conv"] = q_removed
    c["energy_err"] = abs(q_src - q_removed) / (abs(q_src) + 1e-12) if abs(q_src) > 1e-12 else 0.0
    c["energy_pass"] = c["energy_err"] < 0.20
    c["energy_warn"] = c["energy_err"] < 0.40
    return c


def validate(lat, buf: int = 10, core_nx: int | None = None, core_ny: int | None = None, t_inlet: float = 25.0,
             attrs: dict | None = None) -> dict:
    """Checks of the lattice's current fields. Nu, f_friction and Re (u_inlet * D_h / nu, generate_dataset.py:398-400)
    come from the device scalars unless ``attrs`` gives them."""
    nx, ny, nz = lat.shape
    prm = lat.params
    a = {"heat_power": prm["heat_power"], "Pr": prm["Pr"], "k_ratio": prm["k_ratio"], "tau_fluid": prm["tau_fluid"]}
    if attrs is None or not {"Nu", "f_friction", "Re"} <= set(attrs):
        sc = lat.scalars(buf=buf, core_nx=core_nx if core_nx is not None else nx - 2 * buf,
                         core_ny=core_ny if core_ny is not None else ny, t_inlet=t_inlet)
        nu = (prm["tau_fluid"] - 0.5) / 3.0
        a.update(Nu=sc["Nu"], f_friction=sc["f_friction"], Re=prm["u_inlet_val"] * sc["Dh"] / nu)
    if attrs:
        a.update(attrs)
    return checks_from_raw(lat.validate_raw(), a, ny * nz, t_inlet)
