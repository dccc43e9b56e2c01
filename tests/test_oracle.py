"""The oracle itself: pinned by the reference's analytical known-answer tests (validate_analytical.py,
run at the reference's thresholds) and cross-checked against an independent numpy restatement."""
import numpy as np
import pytest

import analytical_cases as A
from oracle import ref_numpy as RN
from oracle.ref import Ref


@pytest.mark.parametrize("name", list(A.CASES))
def test_oracle_passes_reference_analytical_case(name):
    v = A.CASES[name](A.OracleBackend(32))
    assert A.passes(name, v), f"{name}: {v} vs threshold {A.THRESHOLDS[name]}"


def _random_channel(seed, nx=12, ny=9, nz=8, solid_frac=0.2):
    rng = np.random.default_rng(seed)
    m = np.zeros((nx, ny, nz), np.int32)
    m[rng.random((nx, ny, nz)) < solid_frac] = 1
    m[:, 0, :] = 1
    m[:, -1, :] = 1
    m[:, :, 0] = 1
    m[:, :, -1] = 1
    m[0, 1:-1, 1:-1] = 2
    m[-1, 1:-1, 1:-1] = 3
    hs = np.zeros((nx, ny, nz), np.float32)
    hs[:, :, 0] = rng.random((nx, ny)).astype(np.float32)
    return m, hs


@pytest.mark.parametrize("seed", [0, 1])
def test_c_oracle_matches_numpy_twin_bit_for_bit(seed):
    m, hs = _random_channel(seed)
    res = Ref(32).run_simulation(m, max_steps=40, tau_fluid=0.58, heat_power=2e-3, u_inlet_val=0.03, Pr=3.0,
                                 k_ratio=40.0, tol_ke=0, tol_T=0, heat_source=hs, stats_every=1000)
    rho, u, T = RN.run(m, 40, 0.58, 3.0, 40.0, 0.03, 25.0, 2e-3, hs)
    assert np.array_equal(rho, res["rho"]) and np.array_equal(u, res["u"]) and np.array_equal(T, res["T"])


def test_oracle_fp64_close_to_fp32():
    m, hs = _random_channel(3)
    kw = dict(max_steps=200, tau_fluid=0.6, heat_power=1e-3, u_inlet_val=0.04, Pr=2.0, k_ratio=20.0, tol_ke=0,
              tol_T=0, heat_source=hs, stats_every=1000)
    a, b = Ref(32).run_simulation(m, **kw), Ref(64).run_simulation(m, **kw)
    assert np.allclose(a["u"], b["u"], atol=1e-6) and np.allclose(a["T"], b["T"], rtol=1e-5)


def test_oracle_divergence_guard_fires():
    # u_in = 0.3 drives |u| past the 0.17 guard of simulation.py:152
    m, _ = _random_channel(4, solid_frac=0.3)
    res = Ref(32).run_simulation(m, max_steps=2000, tau_fluid=0.52, u_inlet_val=0.3, tol_ke=0, tol_T=0)
    assert res["diverged"] and not res["converged"] and res["steps"] < 2000


def test_oracle_convergence_and_min_steps():
    # simulation.py:104: min_steps = min(0.6*max_steps, max(5000, 2*nx/u_in)) -> 0.6*1000 = 600 here
    m, _ = _random_channel(5, nx=10, ny=6, nz=6, solid_frac=0.0)
    res = Ref(32).run_simulation(m, max_steps=1000, tau_fluid=0.8, u_inlet_val=0.01, tol_ke=1e-3, tol_T=1e-3)
    assert res["converged"] and res["steps"] == 700
