"""The validators' FP64 device reductions (xac_lattice_validate) on a lattice holding the seeded fields, against
the numpy restatement and the reference's checks (tests/golden/validate.json)."""
import json
from pathlib import Path

import pytest
import torch

from oracle.validate_ref import raw_sums
from tests.golden.make_golden import validation_case
from xadvcool_b200.lattice import Lattice
from xadvcool_b200.validate import checks_from_raw, validate

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "validate.json").read_text())


@pytest.mark.parametrize("case", GOLDEN, ids=lambda c: f"seed{c['seed']}")
def test_device_reductions_match(case, cuda):
    mask, rho, u, T, hs, attrs = validation_case(case["seed"])
    lat = Lattice(mask, heat_source=hs, tau_fluid=attrs["tau_fluid"], heat_power=attrs["heat_power"],
                  Pr=attrs["Pr"], k_ratio=attrs["k_ratio"])
    lat.init_fields(torch.from_numpy(rho).cuda(), torch.from_numpy(u).cuda(), torch.from_numpy(T).cuda())
    raw = lat.validate_raw()
    ref = raw_sums(mask, rho, u, T, hs, attrs["heat_power"])
    for k, v in ref.items():
        assert abs(raw[k] - v) <= 1e-6 * max(abs(v), 1e-9), (k, raw[k], v)
    got = validate(lat, attrs=attrs)
    for k, v in case["checks"].items():
        if isinstance(v, bool):
            assert bool(got[k]) == v, k
        else:
            # absolute tolerances for the differences of float32 sums in the reference (see test_validate.py)
            extra = {"delta_P": 1e-6, "mass_err": 1e-6, "energy_err": 1e-5}.get(k, 0.0)
            assert abs(got[k] - v) <= 2e-6 * max(abs(v), 1e-12) + extra, (k, got[k], v)
    lat.close()


def test_validate_after_a_solve(cuda):
    """On real solver output the checks are defined and the flow ones pass for a short, stable run."""
    from xadvcool_b200.designs import straight_fin_plate
    lat = Lattice(straight_fin_plate(), tau_fluid=0.6, u_inlet_val=0.03, heat_power=1e-4)
    lat.step(400)
    c = validate(lat, buf=8, core_nx=48, core_ny=32)
    assert c["mach_pass"] and c["T_lb_warn"]
    assert all(k in c for k in ("mass_err", "energy_err", "mean_div", "delta_P", "f_Re"))
    lat.close()


def test_dataset_writer_from_a_lattice(cuda, tmp_path):
    """A solved lattice written with the reference's schema: the row's scalars are the device scalars and the
    sample's fields are the lattice's fields."""
    import numpy as np
    import pandas as pd
    from xadvcool_b200 import dataset as D
    from xadvcool_b200.designs import gyroid_design
    mask, hs, u_in, info = gyroid_design(2, nx=48, ny=24, nz=16, buf=6)
    u_in = min(u_in, 0.03)  # below the impulsive-start divergence guard
    design = dict(tau_fluid=0.56, u_inlet_val=u_in, heat_power=0.05, heat_source=hs, design_name="gyroid")
    lat = Lattice(mask, heat_source=hs, tau_fluid=0.56, u_inlet_val=u_in, heat_power=0.05)
    res = lat.run(max_steps=300, tol_ke=0.0, tol_T=0.0)
    w = D.DatasetWriter(tmp_path)
    row = w.add_lattice("g2", lat, design, res, elapsed_s=0.1, buf=6)
    w.close()
    sc = lat.scalars(buf=6, core_nx=36, core_ny=24)
    assert row["Nu"] == sc["Nu"] and row["sim_steps"] == res["steps"] and row["grid_cells"] == mask.size
    assert row["converged"] == res["converged"]
    data, attrs = D.load_sample(tmp_path / "samples" / "g2.npz")
    rho, u, T = (t.cpu().numpy() for t in lat.fields())
    assert np.array_equal(data["temperature"], T) and np.array_equal(data["velocity"], u)
    assert pd.read_parquet(tmp_path / "metadata.parquet")["sample_id"].tolist() == ["g2"]
    lat.close()
