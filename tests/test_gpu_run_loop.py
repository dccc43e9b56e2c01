"""xac_lattice_run moves its convergence loop onto the device after the first stats check (one CUDA graph launch
whose while node repeats {stats_every steps, T, stats, decision kernel}). The run must take the same steps,
make the same decisions and end with the same bits as the loop of src/simulation.py:102-156 driven from the
host with Lattice.step / stats / set_inlet."""
import numpy as np
import pytest

from xadvcool_b200 import designs
from xadvcool_b200.lattice import Lattice

pytestmark = pytest.mark.gpu

MAX_V, SUM_KE, MAX_T, SUM_RHO_IN, SUM_RHO_OUT, C_IN, C_OUT, Q_OUT, NONFINITE = 0, 2, 11, 5, 6, 8, 9, 14, 16


def host_run(lat, max_steps, every, tol_ke, tol_T, min_steps, constant_power=False, target_power=1.0):
    prev_ke = prev_max_T = prev_Q = 0.0
    d_ke = dT = 0.0
    dQ = 1.0
    start, step, diverged = lat.steps_done, 0, False
    while step < max_steps:
        chunk = min(every - (start + step) % every, max_steps - step)
        lat.step(chunk)
        step += chunk
        if (start + step) % every:
            continue
        st = lat.stats()
        past = start + step > every
        d_ke = abs(st[SUM_KE] - prev_ke) / (prev_ke + 1e-9) / every if past else 0.0
        dT = abs(st[MAX_T] - prev_max_T) / (prev_max_T + 1e-9) / every if past else 0.0
        dQ = abs(st[Q_OUT] - prev_Q) / (abs(prev_Q) + 1e-12) / every if past else 1.0
        prev_ke, prev_max_T, prev_Q = st[SUM_KE], st[MAX_T], st[Q_OUT]
        if constant_power and start + step > 2000:
            ue = float(np.float32(lat.get_inlet()))
            rin = st[SUM_RHO_IN] / st[C_IN] if st[C_IN] > 0 else 1.0
            rout = st[SUM_RHO_OUT] / st[C_OUT] if st[C_OUT] > 0 else 1.0
            pw = (rin - rout) / 3.0 * (ue * st[C_IN])
            ue = min(max(ue + 0.005 * (target_power - pw), 0.0001), 0.15)
            lat.set_inlet(ue)
        if step > min_steps and d_ke < tol_ke and dT < tol_T and dQ < tol_T:
            break
        if st[NONFINITE] > 0 or st[MAX_V] > 0.17 or st[MAX_T] > 1e4:
            diverged = True
            break
    converged = step > min_steps and d_ke < tol_ke and dT < tol_T and dQ < tol_T
    return {"steps": step, "converged": converged, "diverged": diverged, "d_ke": d_ke, "dT_conv": dT,
            "dQ_conv": dQ, "u_inlet_final": float(np.float32(lat.get_inlet()))}


CASES = {
    # converges on the device, before the step limit
    "converges": dict(max_steps=6000, every=100, tol=1e-2, min_steps=1000, pump=False, u=0.01),
    # runs into the step limit, with a partial last interval
    "limit": dict(max_steps=2550, every=100, tol=1e-12, min_steps=0, pump=False, u=0.01),
    # constant-power pump: the device updates the inlet velocity
    "pump": dict(max_steps=3000, every=100, tol=1e-12, min_steps=0, pump=True, u=0.01),
    # another stats interval
    "every50": dict(max_steps=1500, every=50, tol=1e-5, min_steps=200, pump=False, u=0.01),
    # the divergence guard trips on the device (at step 200, the first check after the host's)
    "diverges": dict(max_steps=3000, every=100, tol=1e-5, min_steps=0, pump=False, u=0.04),
    # 16-bit population storage
    "fp16": dict(max_steps=3000, every=100, tol=1e-3, min_steps=500, pump=False, u=0.01, precision="fp16"),
    "bf16": dict(max_steps=2000, every=100, tol=1e-12, min_steps=0, pump=False, u=0.01, precision="bf16"),
    # a warm start (fields from a short solve): the first step reads them unstreamed, then the device loop
    "warm": dict(max_steps=3000, every=100, tol=1e-3, min_steps=300, pump=False, u=0.01, warm=True),
    # the lattice already advanced 37 steps: the first interval is 63 steps long
    "offset": dict(max_steps=2000, every=100, tol=1e-12, min_steps=0, pump=False, u=0.01, pre=37),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_device_loop_matches_the_host_loop(case, cuda):
    c = CASES[case]
    mask, hs, _, _ = designs.gyroid_design(7, nx=60, ny=32, nz=16)
    kw = dict(heat_source=hs, tau_fluid=0.56, u_inlet_val=c["u"], heat_power=0.05,
              precision=c.get("precision", "fp32"))
    init = None
    if c.get("warm"):
        with Lattice(mask, **kw) as w:
            w.step(400)
            init = [t.clone() for t in w.fields()]
    a = Lattice(mask, **kw)
    if init:
        a.init_fields(*init)
    a.step(c.get("pre", 0))
    got = a.run(max_steps=c["max_steps"], stats_every=c["every"], tol_ke=c["tol"], tol_T=c["tol"],
                min_steps=c["min_steps"], pump_mode="constant_power" if c["pump"] else "constant_flow",
                target_power=0.002)
    b = Lattice(mask, **kw)
    if init:
        b.init_fields(*init)
    b.step(c.get("pre", 0))
    want = host_run(b, c["max_steps"], c["every"], c["tol"], c["tol"], c["min_steps"], constant_power=c["pump"],
                    target_power=0.002)
    for k in ("steps", "converged", "diverged", "d_ke", "dT_conv", "dQ_conv", "u_inlet_final"):
        assert got[k] == want[k], (k, got[k], want[k])
    assert a.steps_done == b.steps_done
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x.cpu().numpy(), y.cpu().numpy())
    assert np.array_equal(a.stats(), b.stats())
    if case == "converges":
        assert got["converged"] and got["steps"] < c["max_steps"], got
    if case == "pump":
        assert got["u_inlet_final"] != pytest.approx(c["u"])
    if case == "diverges":
        assert got["diverged"] and got["steps"] > c["every"], got
    a.close()
    b.close()
