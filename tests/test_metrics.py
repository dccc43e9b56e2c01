"""Scalar outputs (generate_dataset.py:57-179): the numpy restatement is pinned to the reference
function's outputs (tests/golden/metrics.json); the FP64 device reduction is checked against both."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle.metrics_ref import hydraulic_diameter, macroscopic_metrics, porosity
from xadvcool_b200.designs import generate_mask

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))
from make_golden import synthetic_fields  # noqa: E402

CASES = json.loads((GOLD / "metrics.json").read_text())
# the reference accumulates in float32 (numpy pairwise sums); FP64 agrees to this relative tolerance
RTOL = 5e-5


@pytest.mark.parametrize("case", CASES, ids=lambda c: str(c["seed"]))
def test_metric_restatement_matches_reference(case):
    mask = generate_mask(case["state"])
    rho, u, T = synthetic_fields(case["seed"], mask.shape)
    Dh, V, A = hydraulic_diameter(mask)
    assert (Dh, V, A) == (case["Dh"], case["V_fluid"], case["A_wetted"])
    assert porosity(mask) == pytest.approx(case["porosity"], rel=1e-12)
    out = macroscopic_metrics(rho, u, T, mask, case["params"]["tau_fluid"], case["params"]["u_inlet_val"], Dh, A)
    for k, v in case["metrics"].items():
        assert out[k] == pytest.approx(v, rel=RTOL, abs=1e-9), k


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: str(c["seed"]))
def test_device_scalars_match_reference(case, cuda):
    from xadvcool_b200 import metrics
    mask = generate_mask(case["state"])
    rho, u, T = synthetic_fields(case["seed"], mask.shape)
    res = {"rho": rho, "u": u, "T": T}
    out = metrics.compute_macroscopic_metrics(res, mask, case["params"], case["Dh"], case["A_wetted"])
    for k, v in case["metrics"].items():
        assert out[k] == pytest.approx(v, rel=RTOL, abs=1e-9), k
    s = metrics.device_scalars(rho, u, T, mask, tau_fluid=case["params"]["tau_fluid"],
                               u_inlet_val=case["params"]["u_inlet_val"])
    assert s["Dh"] == case["Dh"] and s["A_wetted"] == case["A_wetted"] and s["V_fluid"] == case["V_fluid"]
    assert s["porosity"] == pytest.approx(case["porosity"], rel=1e-12)
    assert s["pressure_drop"] == pytest.approx(case["pressure_drop_all"], rel=1e-5)
    ref64 = macroscopic_metrics(rho, u, T, mask, case["params"]["tau_fluid"], case["params"]["u_inlet_val"],
                                case["Dh"], case["A_wetted"])
    for k in ("R_th", "Q_vol", "T_max_surface", "sigma_T", "delta_P"):
        assert s[k] == pytest.approx(ref64[k], rel=1e-9), k
