"""Physical validators (analyze_dataset.py:184-323). The numpy restatement is pinned to the reference function's
outputs (tests/golden/validate.json); the product's check assembly is tested on numpy-restated reductions here,
and the GPU reductions against the same golden vectors in test_gpu_validate."""
import json
from pathlib import Path

import pytest

from oracle.validate_ref import raw_sums, validate_arrays
from tests.golden.make_golden import validation_case
from xadvcool_b200.validate import checks_from_raw

GOLDEN = json.loads((Path(__file__).parent / "golden" / "validate.json").read_text())


# delta_P, mass_err and energy_err are differences of sums that the reference accumulates over float32 arrays
# (a few float32 ulps of the summed terms, ~1e-7 relative to them): they carry an absolute error of that size,
# not a relative one. Our reductions sum in FP64.
ABS = {"delta_P": 1e-6, "mass_err": 1e-6, "energy_err": 1e-5}


def _close(a, b, rel, key=None):
    if isinstance(b, bool):
        return bool(a) == b
    return abs(a - b) <= rel * max(abs(b), 1e-12) + ABS.get(key, 1e-15)


@pytest.mark.parametrize("case", GOLDEN, ids=lambda c: f"seed{c['seed']}")
def test_oracle_matches_reference(case):
    mask, rho, u, T, hs, attrs = validation_case(case["seed"])
    got = validate_arrays(mask, u, T, rho / 3.0, hs, attrs)
    for k, v in case["checks"].items():
        assert _close(got[k], v, 1e-12), (k, got[k], v)


@pytest.mark.parametrize("case", GOLDEN, ids=lambda c: f"seed{c['seed']}")
def test_checks_from_raw_sums(case):
    mask, rho, u, T, hs, attrs = validation_case(case["seed"])
    raw = raw_sums(mask, rho, u, T, hs, attrs["heat_power"])
    got = checks_from_raw(raw, attrs, mask.shape[1] * mask.shape[2])
    for k, v in case["checks"].items():
        # the reduction sums in FP64 where the reference sums some float32 arrays: a few ulps of float32
        assert _close(got[k], v, 2e-6, k), (k, got[k], v)
