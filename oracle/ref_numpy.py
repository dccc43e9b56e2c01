"""ORACLE — test infrastructure only. A second, independent restatement of the reference kernels in
vectorised numpy (float32, reference layout), for small lattices. It cross-checks the C oracle: numpy
float32 arithmetic rounds every operation, so with the same operand order the two agree bit for bit.
Citations: src/fluid_engine3d.py, src/thermal_engine3d.py (path:line as in the C oracle).
"""
from __future__ import annotations

import numpy as np

BC_FLUID, BC_SOLID, BC_INLET, BC_OUTLET = 0, 1, 2, 3
E = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0],
              [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1], [0, 1, 1],
              [0, -1, -1], [0, 1, -1], [0, -1, 1]], dtype=np.int64)
OPP = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17])
W = np.array([1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12).astype(np.float32)
f32 = np.float32


def _eu(i, ux, uy, uz):
    return f32(E[i, 0]) * ux + f32(E[i, 1]) * uy + f32(E[i, 2]) * uz


def equilibrium(scal, u, mask=None, thermal=False):
    """fluid_engine3d.py:58-80 / thermal_engine3d.py:7-47."""
    ux, uy, uz = u[..., 0].copy(), u[..., 1].copy(), u[..., 2].copy()
    if thermal:
        s = mask == BC_SOLID
        ux[s] = 0
        uy[s] = 0
        uz[s] = 0
    usq = ux * ux + uy * uy + uz * uz
    out = np.empty((19,) + scal.shape, dtype=f32)
    for i in range(19):
        eu = _eu(i, ux, uy, uz)
        out[i] = W[i] * scal * (f32(1.0) + f32(3.0) * eu + f32(4.5) * (eu * eu) - f32(1.5) * usq)
    return out


def macroscopic(f):
    """fluid_engine3d.py:85-113."""
    r = np.zeros(f.shape[1:], f32)
    m = [np.zeros(f.shape[1:], f32) for _ in range(3)]
    for i in range(19):
        r += f[i]
        for k in range(3):
            m[k] += f[i] * f32(E[i, k])
    u = np.zeros(f.shape[1:] + (3,), f32)
    ok = r > f32(1e-10)
    with np.errstate(divide="ignore", invalid="ignore"):
        for k in range(3):
            u[..., k] = np.where(ok, m[k] / r, f32(0.0))
    return r, u


def fused_collision(f_old, rho, u, mask, tau):
    """fluid_engine3d.py:141-176."""
    omega = f32(1.0) / f32(tau)
    fe = equilibrium(rho, u)
    act = mask != BC_SOLID
    return np.where(act[None], f_old - omega * (f_old - fe), f_old).astype(f32)


def streaming(fp, mask, ux_in, rho_out):
    """fluid_engine3d.py:181-272."""
    _, nx, ny, nz = fp.shape
    fs = np.zeros_like(fp)
    ux_in, rho_out = f32(ux_in), f32(rho_out)
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    interior = mask == BC_FLUID
    for i in range(19):
        sx, sy, sz = X - E[i, 0], Y - E[i, 1], Z - E[i, 2]
        oob = (sx < 0) | (sx >= nx) | (sy < 0) | (sy >= ny) | (sz < 0) | (sz >= nz)
        cx, cy, cz = np.clip(sx, 0, nx - 1), np.clip(sy, 0, ny - 1), np.clip(sz, 0, nz - 1)
        bb = oob | (mask[cx, cy, cz] == BC_SOLID)
        v = np.where(bb, fp[OPP[i]], fp[i][cx, cy, cz])
        fs[i][interior] = v[interior]
    inl = mask == BC_INLET
    if inl.any():
        f = {i: fp[i][inl] for i in range(19)}
        rn = (f[0] + f[3] + f[4] + f[5] + f[6] + f[15] + f[16] + f[17] + f[18]
              + f32(2.0) * (f[2] + f[8] + f[10] + f[12] + f[14])) / (f32(1.0) - ux_in)
        c23, c16 = f32(2.0) / f32(3.0), f32(1.0) / f32(6.0)
        new = dict(f)
        new[1] = f[2] + c23 * rn * ux_in
        new[7] = f[10] + c16 * rn * ux_in
        new[9] = f[8] + c16 * rn * ux_in
        new[11] = f[14] + c16 * rn * ux_in
        new[13] = f[12] + c16 * rn * ux_in
        for i in range(19):
            fs[i][inl] = new[i]
    out = np.argwhere(mask == BC_OUTLET)
    for x, y, z in out:
        sx = max(x - 1, 0)
        v = fp[:, sx, y, z].copy()
        s = f32(0.0)
        for i in range(19):
            s = f32(s + v[i])
        if s > f32(1e-6):
            v = v * (rho_out / s)
        fs[:, x, y, z] = v
    # solid destinations keep whatever the output held: the caller passes the previous buffer
    return fs, mask == BC_SOLID


def fused_thermal_collision(g_old, u, T, mask, tau_f, tau_s, hs, power):
    """thermal_engine3d.py:91-145."""
    solid = mask == BC_SOLID
    omega = np.where(solid, f32(1.0) / f32(tau_s), f32(1.0) / f32(tau_f)).astype(f32)
    q = hs.astype(f32) * f32(power)
    ge = equilibrium(T, u, mask, thermal=True)
    out = np.empty_like(g_old)
    srcf = f32(1.0) - f32(0.5) * omega
    for i in range(19):
        v = g_old[i] - omega * (g_old[i] - ge[i])
        out[i] = np.where(q > 0, v + W[i] * srcf * q, v)
    return out


def thermal_streaming(gp, mask, T_in):
    """thermal_engine3d.py:147-211."""
    _, nx, ny, nz = gp.shape
    gs = np.empty_like(gp)
    T_in = f32(T_in)
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    for i in range(19):
        sx, sy, sz = X - E[i, 0], Y - E[i, 1], Z - E[i, 2]
        cx, cy, cz = np.clip(sx, 0, nx - 1), np.clip(sy, 0, ny - 1), np.clip(sz, 0, nz - 1)
        v = gp[i][cx, cy, cz]
        wall = (sy < 0) | (sy >= ny) | (sz < 0) | (sz >= nz)
        v = np.where(wall, gp[OPP[i]], v)
        v = np.where(sx >= nx, gp[i], v)
        v = np.where(sx < 0, W[i] * T_in, v)
        gs[i] = v
    inl, outl = mask == BC_INLET, mask == BC_OUTLET
    for i in range(19):
        gs[i][inl] = W[i] * T_in
        src = np.roll(gp[i], 1, axis=0)
        src[0] = gp[i][0]
        gs[i][outl] = src[outl]
    return gs


def thermal_macroscopic(g):
    T = np.zeros(g.shape[1:], f32)
    for i in range(19):
        T += g[i]
    return T


def run(mask, steps, tau, Pr, k_ratio, u_in, t_in, power, hs=None):
    """src/simulation.py:60-121 for a fixed number of steps (no stats); returns rho, u, T."""
    mask = np.asarray(mask, dtype=np.int32)
    nx, ny, nz = mask.shape
    if hs is None:
        hs = np.zeros(mask.shape, f32)
        hs[:, :, 0] = 1.0
    hs = np.array(hs, dtype=f32)
    if hs.max() > 0:
        hs /= hs.max()
    tth_f = 0.5 + (tau - 0.5) / Pr
    tth_s = 0.5 + k_ratio * (tth_f - 0.5)
    rho = np.ones(mask.shape, f32)
    u = np.zeros(mask.shape + (3,), f32)
    T = np.full(mask.shape, t_in, f32)
    g = equilibrium(T, u, mask, thermal=True)
    f = equilibrium(rho, u)
    for _ in range(steps):
        fp = fused_collision(f, rho, u, mask, tau)
        fs, keep = streaming(fp, mask, u_in, 1.0)
        f = np.where(keep[None], f, fs)
        rho, u = macroscopic(f)
        gp = fused_thermal_collision(g, u, T, mask, tth_f, tth_s, hs, power)
        g = thermal_streaming(gp, mask, t_in)
        T = thermal_macroscopic(g)
    return rho, u, T
