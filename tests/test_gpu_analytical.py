"""The reference's ten analytical validations (validate_analytical.py) on libxac.so's CUDA operators, at the
reference's thresholds, and equal to the oracle's error values."""
import pytest

import analytical_cases as A
from gpu_backend import GpuBackend

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(A.CASES))
def test_cuda_passes_reference_analytical_case(name, cuda):
    v = A.CASES[name](GpuBackend())
    assert A.passes(name, v), f"{name}: {v} vs threshold {A.THRESHOLDS[name]}"
    ref = A.CASES[name](A.OracleBackend(32))
    assert v == pytest.approx(ref, rel=1e-9, abs=1e-9)
