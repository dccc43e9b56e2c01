"""Dataset writer with the reference's schema (generate_dataset.py:488-517 for the per-sample group,
:538-579 for the metadata row), for solves run on this library.

The reference writes one HDF5 group per sample; h5py is not available here, so each sample is one compressed
.npz holding the same five datasets under the same names and dtypes (mask int8, heat_source, velocity,
pressure = rho / 3, temperature) plus the group's attributes as a JSON string. The metadata table is written
as Parquet with the reference's columns.

    w = DatasetWriter("out/")
    w.add_lattice("sample_0001", lat, design, result, elapsed_s)   # after lat.run(...)
    w.close()                                                       # -> out/metadata.parquet

The reference's admission rules decide which solves become samples: ``is_valid_geometry`` before the solve
(generate_dataset.py:281-292), then ``divergence_reason`` and ``plausibility_reason`` after it (:438-483). Their
reason strings are the ones the reference records in failed_samples.json.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

# generate_dataset.py:538-579, in the reference's order
METADATA_COLUMNS = [
    "sample_id", "Pr", "k_ratio", "design_name", "design_idx", "heat_source_type", "feature_size", "spacing",
    "tau_fluid", "u_inlet_val", "heat_power", "porosity", "Dh", "Re", "max_velocity", "max_temperature",
    "mean_temperature", "pressure_drop", "elapsed_s", "sim_steps", "converged", "grid_nx", "grid_ny", "grid_nz",
    "grid_cells", "total_lattice_updates", "mlups", "gpu_name", "R_th", "Nu", "f_friction", "P_pump", "COP",
    "Q_vol", "T_max_surface", "T_avg_surface", "delta_T_max", "sigma_T", "fluid_temp_rise",
]
METRIC_KEYS = ["R_th", "Nu", "f_friction", "P_pump", "COP", "Q_vol", "T_max_surface", "T_avg_surface",
               "delta_T_max", "sigma_T", "fluid_temp_rise"]

# generate_dataset.py:278-279
MIN_POROSITY = 0.15
MAX_POROSITY = 0.90
BC_SOLID = 1


def is_valid_geometry(mask, buf: int = 10):
    """generate_dataset.py:281-292: porosity of the core (x outside the inlet/outlet buffers) within
    [MIN_POROSITY, MAX_POROSITY], and neither the first nor the last core x plane fully solid. Returns
    (valid, porosity); a rejected design is recorded as ``f"invalid geometry (porosity={porosity:.2%})"``."""
    m = np.asarray(mask)
    core = m[buf:-buf, :, :]
    porosity = float(1.0 - np.sum(core == BC_SOLID) / core.size)
    if porosity < MIN_POROSITY or porosity > MAX_POROSITY:
        return False, porosity
    inlet = m[buf, 1:-1, 4:-2]
    outlet = m[-(buf + 1), 1:-1, 4:-2]
    if np.all(inlet == BC_SOLID) or np.all(outlet == BC_SOLID):
        return False, porosity
    return True, porosity


def divergence_reason(u, T):
    """generate_dataset.py:438-447 on the solved fields (reference layout: u (nx,ny,nz,3), T (nx,ny,nz), host
    float32): the reason string, or None when the solve did not diverge."""
    max_v = np.max(np.linalg.norm(np.asarray(u), axis=-1))
    max_T = np.max(np.asarray(T))
    Ma = max_v * (3.0 ** 0.5)
    if np.isnan(max_v) or Ma > 0.3 or np.isnan(max_T) or max_T > 1e4:
        return f"diverged (max_v={max_v:.2e}, Ma={Ma:.2f}, max_T={max_T:.2e})"
    return None


def plausibility_reason(metrics: dict, converged: bool):
    """generate_dataset.py:458-483 on compute_macroscopic_metrics' output and the solve's converged flag: the
    reason string, or None when the sample is kept."""
    Nu, R_th, COP, rise = metrics["Nu"], metrics["R_th"], metrics["COP"], metrics["fluid_temp_rise"]
    reasons = []
    if Nu < 0 or Nu > 2000 or np.isnan(Nu):
        reasons.append(f"Nu={Nu:.1f}")
    if R_th < 0 or R_th > 1000 or np.isnan(R_th):
        reasons.append(f"R_th={R_th:.1f}")
    if COP < 0 or np.isnan(COP):
        reasons.append(f"COP={COP:.2e}")
    if rise < 0 or np.isnan(rise):
        reasons.append(f"fluid_temp_rise={rise:.2e}")
    if not converged:
        reasons.append("not converged")
    return f"unphysical ({', '.join(reasons)})" if reasons else None


def metadata_row(sample_id, design: dict, mask_shape, scalars: dict, steps: int, converged: bool, elapsed_s: float,
                 gpu_name: str = "unknown", Pr: float = 7.0, k_ratio: float = 628.0) -> dict:
    """One row of metadata.parquet. ``design`` carries the run parameters (tau_fluid, u_inlet_val, heat_power)
    and, when known, design_name / design_idx / heat_source_type / feature_size / spacing; ``scalars`` is
    Lattice.scalars() of the converged fields."""
    nx, ny, nz = mask_shape
    nu = (design["tau_fluid"] - 0.5) / 3.0
    cells = int(nx * ny * nz)
    row = {
        "sample_id": sample_id, "Pr": Pr, "k_ratio": k_ratio,
        "design_name": design.get("design_name", ""), "design_idx": design.get("design_idx", -1),
        "heat_source_type": design.get("heat_source_type", ""), "feature_size": design.get("feature_size", 0),
        "spacing": design.get("spacing", 0), "tau_fluid": design["tau_fluid"], "u_inlet_val": design["u_inlet_val"],
        "heat_power": design["heat_power"], "porosity": scalars["porosity"], "Dh": scalars["Dh"],
        "Re": design["u_inlet_val"] * scalars["Dh"] / nu,  # generate_dataset.py:398-400
        "max_velocity": scalars["max_velocity"], "max_temperature": scalars["max_temperature"],
        "mean_temperature": scalars["mean_temperature"],
        "pressure_drop": scalars["pressure_drop"],  # mean over all cells of planes 1 and nx-2 (:556)
        "elapsed_s": elapsed_s, "sim_steps": int(steps), "converged": bool(converged),
        "grid_nx": nx, "grid_ny": ny, "grid_nz": nz, "grid_cells": cells, "total_lattice_updates": cells * int(steps),
        "mlups": cells * int(steps) / (elapsed_s * 1e6) if elapsed_s > 0 else 0.0, "gpu_name": gpu_name,
    }
    row.update({k: scalars[k] for k in METRIC_KEYS})
    return {k: row[k] for k in METADATA_COLUMNS}


def save_sample(path, mask, heat_source, u, rho, T, attrs: dict):
    """The per-sample group of generate_dataset.py:488-517 as a compressed .npz (reference layout fields)."""
    np.savez_compressed(
        path, mask=np.asarray(mask).astype(np.int8), heat_source=np.asarray(heat_source, np.float32),
        velocity=np.asarray(u, np.float32), pressure=(np.asarray(rho, np.float32) / np.float32(3.0)),
        temperature=np.asarray(T, np.float32), attrs=np.array(json.dumps(attrs, default=float)))


def load_sample(path):
    """-> (datasets dict, attrs dict) of a saved sample."""
    with np.load(path) as z:
        data = {k: z[k] for k in ("mask", "heat_source", "velocity", "pressure", "temperature")}
        attrs = json.loads(str(z["attrs"]))
    return data, attrs


class DatasetWriter:
    def __init__(self, out_dir, gpu_name: str | None = None):
        self.dir = Path(out_dir)
        (self.dir / "samples").mkdir(parents=True, exist_ok=True)
        self.rows = []
        if gpu_name is None:
            try:
                import torch
                gpu_name = torch.cuda.get_device_name()
            except Exception:
                gpu_name = "unknown"
        self.gpu_name = gpu_name

    def add(self, sample_id, mask, heat_source, u, rho, T, design: dict, scalars: dict, steps, converged, elapsed_s,
            Pr=7.0, k_ratio=628.0):
        row = metadata_row(sample_id, design, np.shape(mask), scalars, steps, converged, elapsed_s, self.gpu_name,
                           Pr, k_ratio)
        attrs = {k: v for k, v in design.items() if k not in ("mask", "heat_source")}
        attrs.update({k: row[k] for k in METADATA_COLUMNS if k not in ("sample_id",)})
        attrs.update(coolant="water", grid_shape=list(np.shape(mask)))
        hs = heat_source if heat_source is not None else np.zeros(np.shape(mask), np.float32)
        save_sample(self.dir / "samples" / f"{sample_id}.npz", mask, hs, u, rho, T, attrs)
        self.rows.append(row)
        return row

    def add_lattice(self, sample_id, lat, design: dict, result: dict, elapsed_s: float, buf: int = 10,
                    core_nx: int | None = None, core_ny: int | None = None):
        """Fields and scalars of a solved Lattice (after Lattice.run)."""
        nx, ny, nz = lat.shape
        sc = lat.scalars(buf=buf, core_nx=core_nx if core_nx is not None else nx - 2 * buf,
                         core_ny=core_ny if core_ny is not None else ny)
        rho, u, T = (t.cpu().numpy() for t in lat.fields())
        return self.add(sample_id, lat.mask, design.get("heat_source"), u, rho, T, design, sc, result["steps"],
                        result["converged"], elapsed_s, lat.params["Pr"], lat.params["k_ratio"])

    def close(self):
        import pandas as pd
        pd.DataFrame(self.rows, columns=METADATA_COLUMNS).to_parquet(self.dir / "metadata.parquet", index=False)
        return self.dir / "metadata.parquet"
