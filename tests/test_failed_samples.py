"""The reference's admission rules (generate_dataset.py:281-292, :438-483) against its own records: the designs
that dataset/failed_samples.json rejects as invalid geometry are rejected here with the same reason string,
and the designs it admitted (dataset/metadata.parquet rows) pass. Fixtures: tests/golden/failed_rows.json and
parquet_rows.json (see make_golden.py)."""
import json
from pathlib import Path

import numpy as np
import pytest

from xadvcool_b200 import dataset as D
from xadvcool_b200 import designs

GOLD = Path(__file__).resolve().parent / "golden"
FAILED = json.loads((GOLD / "failed_rows.json").read_text())
ROWS = json.loads((GOLD / "parquet_rows.json").read_text())
INVALID = [r for r in FAILED if r["category"] == "invalid geometry"]


def _mask(p):
    return designs.generate_mask({"design_type": p["design_idx"], "feature_size": p["feature_size"],
                                  "spacing": p["spacing"], "buffer_size": 10})


def test_fixture_covers_every_category():
    cats = {r["category"] for r in FAILED}
    assert cats == {"invalid geometry", "diverged", "unphysical"}
    assert len(INVALID) >= 6


@pytest.mark.parametrize("row", INVALID, ids=[r["sample_id"] for r in INVALID])
def test_invalid_geometry_rejected_with_the_reference_reason(row):
    valid, porosity = D.is_valid_geometry(_mask(row["params"]))
    assert not valid
    assert f"invalid geometry (porosity={porosity:.2%})" == row["reason"]


@pytest.mark.parametrize("row", ROWS[::5], ids=[r["sample_id"] for r in ROWS[::5]])
def test_admitted_designs_are_valid(row):
    valid, porosity = D.is_valid_geometry(_mask(row))
    assert valid
    assert porosity == pytest.approx(row["porosity"], abs=1e-12)


def test_blocked_inlet_is_invalid():
    mask = np.zeros((40, 12, 10), np.int32)
    mask[:, :, :2] = 1  # base plate
    valid, _ = D.is_valid_geometry(mask)
    assert valid
    mask[10, 1:-1, 4:-2] = 1  # first core x plane fully solid, porosity still in range
    valid, porosity = D.is_valid_geometry(mask)
    assert not valid and D.MIN_POROSITY < porosity < D.MAX_POROSITY


def test_reason_strings_follow_the_reference_format():
    u = np.zeros((4, 3, 2, 3), np.float32)
    T = np.full((4, 3, 2), 25.0, np.float32)
    assert D.divergence_reason(u, T) is None
    u[1, 1, 1] = (0.2, 0.0, 0.0)
    assert D.divergence_reason(u, T) == "diverged (max_v=2.00e-01, Ma=0.35, max_T=2.50e+01)"
    u[1, 1, 1] = (0.17, 0.0, 0.0)  # stopped by the solver's guard (> 0.17) but Ma <= 0.3: not "diverged"
    assert D.divergence_reason(u, T) is None
    T[0, 0, 0] = np.nan
    assert D.divergence_reason(u, T).startswith("diverged (")
    ok = {"Nu": 10.0, "R_th": 0.1, "COP": 5.0, "fluid_temp_rise": 0.3}
    assert D.plausibility_reason(ok, True) is None
    assert D.plausibility_reason(ok, False) == "unphysical (not converged)"
    assert D.plausibility_reason(dict(ok, R_th=2584180.5), False) == "unphysical (R_th=2584180.5, not converged)"
    assert D.plausibility_reason(dict(ok, Nu=-1.0, COP=-2.0), True) == "unphysical (Nu=-1.0, COP=-2.00e+00)"
