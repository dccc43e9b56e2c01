"""The ten analytical validations of validate_analytical.py, restated against a backend object.

A backend provides arrays (``zeros``, ``full``, ``array``, ``numpy``, ``copy``) and the reference's kernel
names (compute_equilibrium_kernel, bgk_collision_kernel, streaming_kernel, ... and the test-only
periodic / forced / Couette / Dirichlet kernels). The same drivers run on the CPU oracle (numpy arrays)
and on libxac.so's CUDA operators (torch CUDA tensors). Each returns the reference's error measure;
thresholds are the reference's (validate_analytical.py:1174-1223).
"""
from __future__ import annotations

import numpy as np
from scipy.special import erfc

BC_FLUID, BC_SOLID, BC_INLET, BC_OUTLET = 0, 1, 2, 3
THRESHOLDS = {
    "semi_infinite_conduction": 3.0, "rectangular_poiseuille": 3.0, "taylor_green_vortex": 3.0,
    "kuwabara_pin_fin": 5.0, "couette_flow": 3.0, "advection_diffusion_gaussian": 3.0, "conjugate_slab": 3.0,
    "volumetric_heat_source": 3.0, "mach_sensitivity": 5.0, "grid_convergence": 1.8,
}


def semi_infinite_conduction(be):
    """validate_analytical.py:32-113: step change at an inlet plane into a solid bar, vs erfc."""
    nx, ny, nz = 100, 3, 3
    mask = np.full((nx, ny, nz), BC_SOLID, dtype=np.int32)
    mask[0] = BC_INLET
    m = be.array(mask)
    tau = 0.8
    alpha = (1.0 / 3.0) * (tau - 0.5)
    T_s = 100.0
    T = be.full((nx, ny, nz), 0.0)
    u = be.zeros((nx, ny, nz, 3))
    rho = be.full((nx, ny, nz), 1.0)
    g_old, g_new, g_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
    hs = be.zeros((nx, ny, nz))
    be.compute_thermal_equilibrium_kernel(rho, u, T, g_eq, m)
    be.copy(g_old, g_eq)
    steps = 400
    for _ in range(steps):
        be.compute_thermal_equilibrium_kernel(rho, u, T, g_eq, m)
        be.thermal_bgk_collision_kernel(g_old, g_eq, g_new, m, tau, tau, hs, 0.0)
        be.thermal_streaming_kernel(g_new, g_old, m, T_s, nx, ny, nz)
        be.compute_thermal_macroscopic_kernel(g_old, T)
    xs = np.arange(1, 50)
    T_sim = be.numpy(T)[xs, 1, 1]
    T_ana = T_s * erfc(xs / (2.0 * np.sqrt(alpha * steps)))
    return float(np.max(np.abs(T_sim - T_ana) / T_s) * 100.0)


def _poiseuille_shape(Y, Z, a, b, terms=30):
    val = np.zeros_like(Y)
    for i in range(1, terms * 2, 2):
        t1 = ((-1) ** ((i - 1) // 2)) / (i ** 3)
        t2 = 1.0 - np.cosh(i * np.pi * Z / (2 * a)) / np.cosh(i * np.pi * b / (2 * a))
        val += t1 * t2 * np.cos(i * np.pi * Y / (2 * a))
    return val


def rectangular_poiseuille(be):
    """validate_analytical.py:116-252: duct flow from the velocity inlet to the pressure outlet; Fourier
    solution scaled by the measured pressure gradient."""
    nx, ny, nz = 60, 21, 11
    mask = np.full((nx, ny, nz), BC_FLUID, dtype=np.int32)
    mask[:, 0, :] = BC_SOLID
    mask[:, -1, :] = BC_SOLID
    mask[:, :, 0] = BC_SOLID
    mask[:, :, -1] = BC_SOLID
    mask[0, 1:-1, 1:-1] = BC_INLET
    mask[-1, 1:-1, 1:-1] = BC_OUTLET
    m = be.array(mask)
    tau, u_in = 0.6, 0.01
    u_inlet = be.array(np.array([u_in], dtype=np.float32))
    rho = be.full((nx, ny, nz), 1.0)
    u = be.zeros((nx, ny, nz, 3))
    f_old, f_new, f_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
    be.compute_equilibrium_kernel(rho, u, f_eq)
    be.copy(f_old, f_eq)
    for _ in range(4000):
        be.bgk_collision_kernel(f_old, f_eq, f_new, m, tau)
        be.streaming_kernel(f_new, f_old, m, u_inlet, 1.0, nx, ny, nz)
        be.compute_macroscopic_kernel(f_old, rho, u)
        be.compute_equilibrium_kernel(rho, u, f_eq)
    u_np, rho_np = be.numpy(u), be.numpy(rho)
    u_slice = u_np[nx - 10, :, :, 0]
    w, h = ny - 2, nz - 2
    a, b = w / 2.0, h / 2.0
    uc = np.max(u_slice)
    Y, Z = np.meshgrid(np.linspace(-w / 2 + 0.5, w / 2 - 0.5, w), np.linspace(-h / 2 + 0.5, h / 2 - 0.5, h),
                       indexing="ij")
    shape = _poiseuille_shape(Y, Z, a, b)
    nu = (1.0 / 3.0) * (tau - 0.5)
    x1, x2 = 10, nx - 15
    dpdx = (1.0 / 3.0) * (np.mean(rho_np[x2, 1:-1, 1:-1]) - np.mean(rho_np[x1, 1:-1, 1:-1])) / float(x2 - x1)
    u_ana = (-dpdx) * (16.0 * a ** 2 / np.pi ** 3) * shape / nu
    return float(np.max(np.abs(u_slice[1:-1, 1:-1] - u_ana) / uc) * 100.0)


def _tgv_fields(nx, ny, nz, U0, k, cs2=1.0 / 3.0):
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    u = np.zeros((nx, ny, nz, 3), dtype=np.float32)
    rho = np.zeros((nx, ny, nz), dtype=np.float32)
    for z in range(nz):
        u[:, :, z, 0] = U0 * np.sin(k * X) * np.cos(k * Y)
        u[:, :, z, 1] = -U0 * np.cos(k * X) * np.sin(k * Y)
        rho[:, :, z] = 1.0 - (U0 ** 2 / (4.0 * cs2)) * (np.cos(2 * k * X) + np.cos(2 * k * Y))
    return X, Y, u, rho


def taylor_green_vortex(be):
    """validate_analytical.py:275-374: periodic vortex, kinetic energy decay exp(-4 nu k^2 t)."""
    L = 32
    nx, ny, nz = L, L, 2
    tau, U0 = 0.55, 0.05
    nu = (tau - 0.5) / 3.0
    k = 2.0 * np.pi / L
    _, _, u_np, rho_np = _tgv_fields(nx, ny, nz, U0, k)
    u, rho = be.array(u_np), be.array(rho_np)
    f_old, f_new, f_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
    m = be.array(np.full((nx, ny, nz), BC_FLUID, dtype=np.int32))
    be.compute_equilibrium_kernel(rho, u, f_eq)
    be.copy(f_old, f_eq)
    ke0 = 0.5 * np.sum(u_np[..., 0] ** 2 + u_np[..., 1] ** 2)
    kes = [ke0]
    for s in range(1, 1001):
        be.bgk_collision_kernel(f_old, f_eq, f_new, m, tau)
        be.periodic_streaming_kernel(f_new, f_old, nx, ny, nz)
        be.compute_macroscopic_kernel(f_old, rho, u)
        be.compute_equilibrium_kernel(rho, u, f_eq)
        if s % 100 == 0:
            uc = be.numpy(u)
            kes.append(0.5 * np.sum(uc[..., 0] ** 2 + uc[..., 1] ** 2))
    t = np.arange(0, 1001, 100)
    ana = ke0 * np.exp(-4.0 * nu * k ** 2 * t)
    return float(np.max(np.abs(np.array(kes) - ana) / ke0) * 100.0)


def kuwabara_pin_fin(be):
    """validate_analytical.py:422-499: body-force flow through a periodic cylinder array vs Kuwabara."""
    L, R = 40, 8.0
    nx, ny, nz = L, L, 3
    xx, yy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    cyl = (xx - L / 2.0) ** 2 + (yy - L / 2.0) ** 2 <= R ** 2
    mask = np.full((nx, ny, nz), BC_FLUID, dtype=np.int32)
    for z in range(nz):
        mask[cyl, z] = BC_SOLID
    m = be.array(mask)
    tau, F = 0.8, 1e-5
    nu = (tau - 0.5) / 3.0
    rho = be.full((nx, ny, nz), 1.0)
    u = be.zeros((nx, ny, nz, 3))
    f_old, f_new, f_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
    be.compute_equilibrium_kernel(rho, u, f_eq)
    be.copy(f_old, f_eq)
    for _ in range(4000):
        be.forced_bgk_collision_kernel(f_old, f_eq, f_new, m, tau, F)
        be.periodic_streaming_with_solids_kernel(f_new, f_old, m, nx, ny, nz)
        be.compute_macroscopic_kernel(f_old, rho, u)
        be.compute_equilibrium_kernel(rho, u, f_eq)
    U = np.mean(be.numpy(u)[:, :, 1, 0])
    phi = float(np.sum(cyl)) / float(nx * ny)
    K = -0.5 * np.log(phi) - 0.75 + phi - 0.25 * phi ** 2
    U_ana = F * L ** 2 * K / (4.0 * np.pi * nu)
    return float(abs(U - U_ana) / U_ana * 100.0)


def couette_flow(be):
    """validate_analytical.py:540-604: moving lid at z >= nz, linear profile."""
    nx, ny, nz = 5, 5, 21
    m = be.array(np.full((nx, ny, nz), BC_FLUID, dtype=np.int32))
    tau, uw = 0.6, 0.05
    rho = be.full((nx, ny, nz), 1.0)
    u = be.zeros((nx, ny, nz, 3))
    f_old, f_new, f_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
    be.compute_equilibrium_kernel(rho, u, f_eq)
    be.copy(f_old, f_eq)
    for _ in range(20000):
        be.bgk_collision_kernel(f_old, f_eq, f_new, m, tau)
        be.couette_streaming_kernel(f_new, f_old, m, uw, nx, ny, nz)
        be.compute_macroscopic_kernel(f_old, rho, u)
        be.compute_equilibrium_kernel(rho, u, f_eq)
    prof = be.numpy(u)[2, 2, :, 0]
    ana = uw * (np.arange(nz) + 0.5) / float(nz)
    return float(np.max(np.abs(prof - ana) / uw) * 100.0)


def advection_diffusion_gaussian(be):
    """validate_analytical.py:623-708: advected, diffusing Gaussian; mean and variance."""
    nx, ny, nz = 200, 3, 3
    tau = 0.8
    alpha = (1.0 / 3.0) * (tau - 0.5)
    U0, x0, s0 = 0.05, 50.0, 10.0
    u_np = np.zeros((nx, ny, nz, 3), dtype=np.float32)
    u_np[..., 0] = U0
    xs = np.arange(nx, dtype=float)
    T_np = np.zeros((nx, ny, nz), dtype=np.float32)
    T_np[:] = np.exp(-((xs - x0) ** 2) / (2.0 * s0))[:, None, None]
    rho = be.full((nx, ny, nz), 1.0)
    u, T = be.array(u_np), be.array(T_np)
    g_old, g_new, g_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
    m = be.array(np.full((nx, ny, nz), BC_FLUID, dtype=np.int32))
    hs = be.zeros((nx, ny, nz))
    be.compute_thermal_equilibrium_kernel(rho, u, T, g_eq, m)
    be.copy(g_old, g_eq)
    steps = 1000
    for _ in range(steps):
        be.thermal_bgk_collision_kernel(g_old, g_eq, g_new, m, tau, tau, hs, 0.0)
        be.periodic_thermal_streaming_kernel(g_new, g_old, nx, ny, nz)
        be.compute_thermal_macroscopic_kernel(g_old, T)
        be.compute_thermal_equilibrium_kernel(rho, u, T, g_eq, m)
    Tf = be.numpy(T)[:, 1, 1].astype(np.float64)
    pdf = Tf / np.sum(Tf)
    mean = np.sum(xs * pdf)
    var = np.sum((xs - mean) ** 2 * pdf)
    var_a, mean_a = s0 + 2.0 * alpha * steps, x0 + U0 * steps
    return float(max(abs(mean - mean_a) / mean_a, abs(var - var_a) / var_a) * 100.0)


def conjugate_slab(be):
    """validate_analytical.py:711-832: solid/fluid slab, piecewise linear steady profile (flux continuity)."""
    nx, ny, nz = 100, 3, 3
    xi = nx // 2
    tau_s, tau_f = 0.8, 0.6
    a_s, a_f = (tau_s - 0.5) / 3.0, (tau_f - 0.5) / 3.0
    T_hot, T_cold = 100.0, 0.0
    mask = np.full((nx, ny, nz), BC_FLUID, dtype=np.int32)
    mask[:xi] = BC_SOLID
    mask[0] = BC_INLET
    mask[-1] = BC_INLET
    m = be.array(mask)
    Ls, Lf = float(xi), float(nx - xi)
    Ti = (a_s * T_hot * Lf + a_f * T_cold * Ls) / (a_s * Lf + a_f * Ls)
    prof = np.array([T_hot + (Ti - T_hot) * (i / Ls) if i < xi else Ti + (T_cold - Ti) * ((i - xi) / Lf)
                     for i in range(nx)])
    T_init = np.zeros((nx, ny, nz), dtype=np.float32)
    T_init[:] = prof[:, None, None]
    T = be.array(T_init)
    u = be.zeros((nx, ny, nz, 3))
    rho = be.full((nx, ny, nz), 1.0)
    g_old, g_new, g_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
    hs = be.zeros((nx, ny, nz))
    be.compute_thermal_equilibrium_kernel(rho, u, T, g_eq, m)
    be.copy(g_old, g_eq)
    for _ in range(30000):
        be.compute_thermal_equilibrium_kernel(rho, u, T, g_eq, m)
        be.thermal_bgk_collision_kernel(g_old, g_eq, g_new, m, tau_f, tau_s, hs, 0.0)
        be.thermal_streaming_kernel(g_new, g_old, m, T_cold, nx, ny, nz)
        be.dirichlet_thermal_bc_kernel(g_old, T_hot, 0, ny, nz)
        be.compute_thermal_macroscopic_kernel(g_old, T)
    T_sim = be.numpy(T)[:, 1, 1]
    sl = slice(2, nx - 2)
    return float(np.max(np.abs(T_sim[sl] - prof[sl]) / (T_hot - T_cold)) * 100.0)


def volumetric_heat_source(be):
    """validate_analytical.py:835-936: uniformly heated solid rod between two Dirichlet planes, parabola."""
    nx, ny, nz = 52, 17, 17
    tau = 0.8
    alpha = (tau - 0.5) / 3.0
    Q = 0.001
    mask = np.full((nx, ny, nz), BC_SOLID, dtype=np.int32)
    mask[0] = BC_INLET
    mask[-1] = BC_INLET
    m = be.array(mask)
    T = be.full((nx, ny, nz), 0.0)
    u = be.zeros((nx, ny, nz, 3))
    rho = be.full((nx, ny, nz), 1.0)
    g_old, g_new, g_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
    hs_np = np.zeros((nx, ny, nz), dtype=np.float32)
    hs_np[1:-1] = 1.0
    hs = be.array(hs_np)
    be.compute_thermal_equilibrium_kernel(rho, u, T, g_eq, m)
    be.copy(g_old, g_eq)
    for _ in range(40000):
        be.compute_thermal_equilibrium_kernel(rho, u, T, g_eq, m)
        be.thermal_bgk_collision_kernel(g_old, g_eq, g_new, m, tau, tau, hs, Q)
        be.thermal_streaming_kernel(g_new, g_old, m, 0.0, nx, ny, nz)
        be.compute_thermal_macroscopic_kernel(g_old, T)
    T_sim = be.numpy(T)[:, ny // 2, nz // 2]
    Q_eff = (1.0 - 0.5 / tau) * Q
    L = float(nx - 1)
    T_max = Q_eff * L ** 2 / (8.0 * alpha)
    xs = np.arange(nx, dtype=float)
    ana = (Q_eff / (2.0 * alpha)) * xs * (L - xs)
    sl = slice(2, nx - 2)
    return float(np.max(np.abs(T_sim[sl] - ana[sl]) / T_max) * 100.0)


def mach_sensitivity(be):
    """validate_analytical.py:939-1039: TGV at five Mach numbers, worst L2 velocity error in percent."""
    L = 64
    nx, ny, nz = L, L, 2
    tau = 0.55
    nu = (tau - 0.5) / 3.0
    k = 2.0 * np.pi / L
    steps = 500
    worst = 0.0
    for U0 in (0.005, 0.01, 0.02, 0.05, 0.1):
        X, Y, u_np, rho_np = _tgv_fields(nx, ny, nz, U0, k)
        u, rho = be.array(u_np), be.array(rho_np)
        f_old, f_new, f_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
        m = be.array(np.full((nx, ny, nz), BC_FLUID, dtype=np.int32))
        be.compute_equilibrium_kernel(rho, u, f_eq)
        be.copy(f_old, f_eq)
        for _ in range(steps):
            be.bgk_collision_kernel(f_old, f_eq, f_new, m, tau)
            be.periodic_streaming_kernel(f_new, f_old, nx, ny, nz)
            be.compute_macroscopic_kernel(f_old, rho, u)
            be.compute_equilibrium_kernel(rho, u, f_eq)
        d = np.exp(-2.0 * nu * k ** 2 * steps)
        ux_a = U0 * np.sin(k * X) * np.cos(k * Y) * d
        uy_a = -U0 * np.cos(k * X) * np.sin(k * Y) * d
        us = be.numpy(u)
        num = np.sqrt(np.mean((us[:, :, 0, 0] - ux_a) ** 2 + (us[:, :, 0, 1] - uy_a) ** 2))
        den = np.sqrt(np.mean(ux_a ** 2 + uy_a ** 2))
        worst = max(worst, num / den * 100.0)
    return float(worst)


def grid_convergence(be):
    """validate_analytical.py:1042-1162: body-force channel at ny in {5,9,13,17}, observed order."""
    nx, nz, tau, umax = 5, 3, 0.8, 0.01
    nu = (tau - 0.5) / 3.0
    errs, dxs = [], []
    for ny in (5, 9, 13, 17):
        a = (ny - 2) / 2.0
        F = 2.0 * nu * umax / a ** 2
        steps = int(20.0 * a ** 2 / nu) + 3000
        mask = np.full((nx, ny, nz), BC_FLUID, dtype=np.int32)
        mask[:, 0, :] = BC_SOLID
        mask[:, -1, :] = BC_SOLID
        m = be.array(mask)
        rho = be.full((nx, ny, nz), 1.0)
        u = be.zeros((nx, ny, nz, 3))
        f_old, f_new, f_eq = (be.zeros((19, nx, ny, nz)) for _ in range(3))
        be.compute_equilibrium_kernel(rho, u, f_eq)
        be.copy(f_old, f_eq)
        for _ in range(steps):
            be.forced_bgk_collision_kernel(f_old, f_eq, f_new, m, tau, F)
            be.periodic_streaming_with_solids_kernel(f_new, f_old, m, nx, ny, nz)
            be.compute_macroscopic_kernel(f_old, rho, u)
            be.compute_equilibrium_kernel(rho, u, f_eq)
        ux = be.numpy(u)[nx - 2, :, 1, 0] + F / 2.0
        yc = (ny - 1) / 2.0
        ana = umax * (1.0 - ((np.arange(ny) - yc) / a) ** 2)
        sl = slice(1, ny - 1)
        num = np.sqrt(np.mean((ux[sl] - ana[sl]) ** 2))
        den = np.sqrt(np.mean(ana[sl] ** 2))
        errs.append(num / den if den >= 1e-10 else num)
        dxs.append(1.0 / (ny - 1))
    ps = [np.log(errs[i] / errs[i + 1]) / np.log(dxs[i] / dxs[i + 1]) for i in range(len(errs) - 1)
          if errs[i + 1] > 1e-10]
    return float(np.mean(ps)) if ps else 0.0


CASES = {
    "semi_infinite_conduction": semi_infinite_conduction,
    "rectangular_poiseuille": rectangular_poiseuille,
    "taylor_green_vortex": taylor_green_vortex,
    "kuwabara_pin_fin": kuwabara_pin_fin,
    "couette_flow": couette_flow,
    "advection_diffusion_gaussian": advection_diffusion_gaussian,
    "conjugate_slab": conjugate_slab,
    "volumetric_heat_source": volumetric_heat_source,
    "mach_sensitivity": mach_sensitivity,
    "grid_convergence": grid_convergence,
}


def passes(name: str, value: float) -> bool:
    thr = THRESHOLDS[name]
    return value >= thr if name == "grid_convergence" else value <= thr


class OracleBackend:
    """Numpy arrays + the C oracle (float32)."""

    def __init__(self, bits=32):
        from oracle.ref import Ref
        self.r = Ref(bits)
        self.dt = self.r.dtype

    def zeros(self, shape):
        return np.zeros(shape, dtype=self.dt)

    def full(self, shape, v):
        return np.full(shape, v, dtype=self.dt)

    def array(self, a):
        a = np.asarray(a)
        if a.dtype == np.int32:
            return np.ascontiguousarray(a)
        return np.ascontiguousarray(a, dtype=self.dt)

    def numpy(self, a):
        return np.asarray(a)

    def copy(self, dst, src):
        dst[...] = src

    def __getattr__(self, name):
        return getattr(self.r, name)
