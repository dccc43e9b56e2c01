"""Dataset writer: the reference's metadata columns (generate_dataset.py:538-579) and per-sample group
(:488-517), round trips through Parquet and .npz, and the reference validators reading a written sample."""
import json
from pathlib import Path

import numpy as np
import pandas as pd

from oracle.validate_ref import validate_arrays
from tests.golden.make_golden import validation_case
from xadvcool_b200 import dataset as D

HERE = Path(__file__).parent


def _scalars(seed):
    rng = np.random.default_rng(seed)
    keys = D.METRIC_KEYS + ["porosity", "Dh", "max_velocity", "max_temperature", "mean_temperature",
                            "pressure_drop"]
    return {k: float(rng.uniform(0.1, 2.0)) for k in keys}


def test_columns_cover_the_reference_metadata():
    rows = json.loads((HERE / "golden" / "parquet_rows.json").read_text())
    # columns the fixture script adds for its own checks, not part of the reference's table
    added = {"mask_sha256", "Dh_check", "porosity_check", "V_fluid", "A_wetted"}
    ref_cols = set(rows[0]) - added
    assert ref_cols <= set(D.METADATA_COLUMNS), ref_cols - set(D.METADATA_COLUMNS)
    assert len(D.METADATA_COLUMNS) == len(set(D.METADATA_COLUMNS)) == 39


def test_round_trip(tmp_path):
    w = D.DatasetWriter(tmp_path, gpu_name="test")
    rows = []
    for seed in range(2):
        mask, rho, u, T, hs, attrs = validation_case(seed)
        design = {"tau_fluid": attrs["tau_fluid"], "u_inlet_val": 0.03, "heat_power": attrs["heat_power"],
                  "design_name": "gyroid", "design_idx": seed, "heat_source_type": "gaussian_hotspots"}
        rows.append(w.add(f"s{seed}", mask, hs, u, rho, T, design, _scalars(seed), 1200 + seed, True, 0.5))
    path = w.close()
    df = pd.read_parquet(path)
    assert list(df.columns) == D.METADATA_COLUMNS
    assert len(df) == 2 and df["sample_id"].tolist() == ["s0", "s1"]
    assert df["total_lattice_updates"].tolist() == [r["grid_cells"] * r["sim_steps"] for r in rows]
    nu = (0.55 - 0.5) / 3.0
    assert np.isclose(df["Re"][0], 0.03 * rows[0]["Dh"] / nu)
    data, a = D.load_sample(tmp_path / "samples" / "s1.npz")
    mask, rho, u, T, hs, attrs = validation_case(1)
    assert data["mask"].dtype == np.int8 and np.array_equal(data["mask"], mask)
    assert np.array_equal(data["velocity"], u) and np.array_equal(data["temperature"], T)
    assert np.array_equal(data["pressure"], rho / np.float32(3.0))
    assert a["coolant"] == "water" and a["grid_shape"] == list(mask.shape) and a["sim_steps"] == 1201
    # the reference's validators read a written sample the way they read an HDF5 group
    c = validate_arrays(data["mask"], data["velocity"], data["temperature"], data["pressure"], data["heat_source"],
                        dict(attrs, Nu=a["Nu"], f_friction=a["f_friction"], Re=a["Re"]))
    assert np.isfinite(c["mass_err"]) and np.isfinite(c["energy_err"])
