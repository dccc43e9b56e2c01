"""Drop-in for src/simulation.py: ``run_simulation`` with the reference's signature and return dict,
running the fused coupled step of libxac.so on a B200."""
from __future__ import annotations

import numpy as np

from .lattice import Lattice, derived_taus  # noqa: F401


def run_simulation(mask,
                   max_steps=40000,
                   tau_fluid=0.52,
                   heat_power=0.1,
                   t_inlet=25.0,
                   u_inlet_val=0.03,
                   stats_every=100,
                   tol_ke=1e-7,
                   tol_T=1e-7,
                   pump_mode="constant_flow",
                   target_power=1.0,
                   device="cuda",
                   silent=False,
                   heat_source=None,
                   Pr=7.0,
                   k_ratio=628.0,
                   *,
                   precision="fp32",
                   init_fields=None,
                   keep_lattice=False,
                   min_steps=0):
    """src/simulation.py:14-162. Same arguments and the same returned keys
    (u, rho, T as numpy float32 in the reference layout, mask, steps, d_ke, dT_conv, dQ_conv, converged).

    Extra keyword-only arguments: ``precision`` (population storage: "fp32"; "fp16" in both
    lattices; "bf16" fluid with FP16 thermal populations; "fp32_t16" FP32 fluid with FP16 thermal populations),
    ``init_fields`` = (rho, u, T) CUDA tensors to warm-start from, ``keep_lattice`` to also return the
    live :class:`Lattice` under key "lattice" (for device-side scalars), ``min_steps`` > 0 to replace the
    reference's minimum run length before convergence (for warm starts).
    """
    nx, ny, nz = np.shape(mask)
    if not silent:
        print(f"Simulation Domain: {nx}x{ny}x{nz}")
    lat = Lattice(mask, tau_fluid=tau_fluid, heat_power=heat_power, t_inlet=t_inlet, u_inlet_val=u_inlet_val,
                  heat_source=heat_source, Pr=Pr, k_ratio=k_ratio, precision=precision, device=device)
    if init_fields is not None:
        lat.init_fields(*init_fields)
    res = lat.run(max_steps=max_steps, stats_every=stats_every, tol_ke=tol_ke, tol_T=tol_T, pump_mode=pump_mode,
                  target_power=target_power, min_steps=min_steps)
    if res["diverged"] and not silent:
        st = res["last_stats"]
        max_v, max_T = st[0], st[11]
        print(f"\n⚠ Simulation diverged at step {res['steps']}: MaxV={max_v:.2e}, Ma={max_v * 3.0 ** 0.5:.2f}, "
              f"MaxT={max_T:.2e}")
    rho, u, T = lat.fields()
    out = {"u": u.cpu().numpy(), "rho": rho.cpu().numpy(), "T": T.cpu().numpy(), "mask": mask,
           "steps": res["steps"], "d_ke": res["d_ke"], "dT_conv": res["dT_conv"], "dQ_conv": res["dQ_conv"],
           "converged": res["converged"]}
    if keep_lattice:
        out["lattice"] = lat
    else:
        lat.close()
    return out
