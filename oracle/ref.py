"""ORACLE — test infrastructure only. ctypes wrapper of liblbm_ref.so (oracle/lbm_ref.c), the C
restatement of the reference's kernels, in the reference layout on numpy arrays.

``Ref(32)`` wraps the float32 build (parity oracle), ``Ref(64)`` the float64 build. Every method is named
after the reference kernel it restates (src/fluid_engine3d.py, src/thermal_engine3d.py,
validate_analytical.py); ``run_simulation`` restates src/simulation.py:14-162.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liblbm_ref.so"


def build() -> Path:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def threads() -> int:
    f = lib().ref_num_threads
    f.restype = C.c_int
    return int(f())


class Ref:
    def __init__(self, bits: int = 32):
        if bits not in (32, 64):
            raise ValueError("bits must be 32 or 64")
        self.bits = bits
        self.dtype = np.float32 if bits == 32 else np.float64
        self._pfx = f"ref{bits}_"
        self.R = C.c_float if bits == 32 else C.c_double

    # -- helpers ------------------------------------------------------------------------------
    def _fn(self, name):
        return getattr(lib(), self._pfx + name)

    def _arr(self, a, shape=None):
        a = np.asarray(a)
        if a.dtype != self.dtype or not a.flags.c_contiguous:
            raise TypeError(f"expected a C-contiguous {self.dtype} array")
        if shape is not None and a.shape != tuple(shape):
            raise ValueError(f"expected shape {shape}, got {a.shape}")
        return _p(a)

    @staticmethod
    def _mask(m):
        m = np.asarray(m)
        if m.dtype != np.int32 or not m.flags.c_contiguous:
            raise TypeError("mask must be a C-contiguous int32 array")
        return _p(m)

    def zeros(self, shape):
        return np.zeros(shape, dtype=self.dtype)

    # -- src/fluid_engine3d.py ---------------------------------------------------------------------
    def compute_equilibrium_kernel(self, rho, u, f_eq):
        nx, ny, nz = rho.shape
        self._fn("equilibrium")(self._arr(rho), self._arr(u), self._arr(f_eq), nx, ny, nz)

    def compute_macroscopic_kernel(self, f, rho, u):
        _, nx, ny, nz = f.shape
        self._fn("macroscopic")(self._arr(f), self._arr(rho), self._arr(u), nx, ny, nz)

    def bgk_collision_kernel(self, f_old, f_eq, f_post, mask, tau):
        _, nx, ny, nz = f_old.shape
        self._fn("bgk_collision")(self._arr(f_old), self._arr(f_eq), self._arr(f_post), self._mask(mask),
                                  self.R(tau), nx, ny, nz)

    def fused_equilibrium_collision_kernel(self, f_old, rho, u, f_post, mask, tau):
        _, nx, ny, nz = f_old.shape
        self._fn("fused_collision")(self._arr(f_old), self._arr(rho), self._arr(u), self._arr(f_post),
                                    self._mask(mask), self.R(tau), nx, ny, nz)

    def streaming_kernel(self, f_post, f_streamed, mask, u_inlet, rho_outlet, nx, ny, nz):
        u_in = float(np.asarray(u_inlet).reshape(-1)[0])
        self._fn("streaming")(self._arr(f_post), self._arr(f_streamed), self._mask(mask), self.R(u_in),
                              self.R(rho_outlet), nx, ny, nz)

    # -- src/thermal_engine3d.py -------------------------------------------------------------------
    def compute_thermal_equilibrium_kernel(self, rho, u, T, g_eq, mask):
        nx, ny, nz = T.shape
        self._fn("thermal_equilibrium")(self._arr(u), self._arr(T), self._arr(g_eq), self._mask(mask), nx, ny, nz)

    def thermal_bgk_collision_kernel(self, g_old, g_eq, g_new, mask, tau_f, tau_s, hs, power):
        _, nx, ny, nz = g_old.shape
        self._fn("thermal_bgk_collision")(self._arr(g_old), self._arr(g_eq), self._arr(g_new), self._mask(mask),
                                          self.R(tau_f), self.R(tau_s), self._arr(hs), self.R(power), nx, ny, nz)

    def fused_thermal_equilibrium_collision_kernel(self, g_old, u, T, g_new, mask, tau_f, tau_s, hs, power):
        _, nx, ny, nz = g_old.shape
        self._fn("fused_thermal_collision")(self._arr(g_old), self._arr(u), self._arr(T), self._arr(g_new),
                                            self._mask(mask), self.R(tau_f), self.R(tau_s), self._arr(hs),
                                            self.R(power), nx, ny, nz)

    def thermal_streaming_kernel(self, g_post, g_streamed, mask, T_inlet, nx, ny, nz):
        self._fn("thermal_streaming")(self._arr(g_post), self._arr(g_streamed), self._mask(mask), self.R(T_inlet),
                                      nx, ny, nz)

    def compute_thermal_macroscopic_kernel(self, g, T):
        _, nx, ny, nz = g.shape
        self._fn("thermal_macroscopic")(self._arr(g), self._arr(T), nx, ny, nz)

    def stats(self, rho, u, T, mask) -> np.ndarray:
        nx, ny, nz = rho.shape
        out = np.zeros(17, dtype=np.float64)
        self._fn("stats")(self._arr(rho), self._arr(u), self._arr(T), self._mask(mask), _p(out), nx, ny, nz)
        return out

    # -- validate_analytical.py test-only kernels ------------------------------------------------
    def dirichlet_thermal_bc_kernel(self, g, T_val, x_plane, ny, nz):
        _, nx, _, _ = g.shape
        self._fn("dirichlet_thermal_plane")(self._arr(g), self.R(T_val), int(x_plane), nx, ny, nz)

    def periodic_streaming_kernel(self, f_post, f_streamed, nx, ny, nz):
        self._fn("periodic_streaming")(self._arr(f_post), self._arr(f_streamed), nx, ny, nz)

    periodic_thermal_streaming_kernel = periodic_streaming_kernel

    def forced_bgk_collision_kernel(self, f_old, f_eq, f_new, mask, tau, force_x):
        _, nx, ny, nz = f_old.shape
        self._fn("forced_bgk_collision")(self._arr(f_old), self._arr(f_eq), self._arr(f_new), self._mask(mask),
                                         self.R(tau), self.R(force_x), nx, ny, nz)

    def periodic_streaming_with_solids_kernel(self, f_post, f_streamed, mask, nx, ny, nz):
        self._fn("periodic_streaming_solids")(self._arr(f_post), self._arr(f_streamed), self._mask(mask), nx, ny, nz)

    def couette_streaming_kernel(self, f_post, f_streamed, mask, u_wall_x, nx, ny, nz):
        self._fn("couette_streaming")(self._arr(f_post), self._arr(f_streamed), self._mask(mask), self.R(u_wall_x),
                                      nx, ny, nz)

    # -- src/simulation.py --------------------------------------------------------------------------
    def run_simulation(self, mask, max_steps=40000, tau_fluid=0.52, heat_power=0.1, t_inlet=25.0, u_inlet_val=0.03,
                       stats_every=100, tol_ke=1e-7, tol_T=1e-7, pump_mode="constant_flow", target_power=1.0,
                       heat_source=None, Pr=7.0, k_ratio=628.0, init_fields=None):
        mask = np.ascontiguousarray(mask, dtype=np.int32)
        nx, ny, nz = mask.shape
        # src/simulation.py:77-86 (normalisation in float32, as numpy does there)
        if heat_source is not None:
            hs = np.array(heat_source, dtype=np.float32)
            if hs.shape != (nx, ny, nz):
                raise ValueError(f"heat_source shape {hs.shape} != domain shape ({nx}, {ny}, {nz})")
        else:
            hs = np.zeros((nx, ny, nz), dtype=np.float32)
            hs[:, :, 0] = 1.0
        if hs.max() > 0:
            hs /= hs.max()
        hs = np.ascontiguousarray(hs.astype(self.dtype))
        rho = np.zeros((nx, ny, nz), self.dtype)
        u = np.zeros((nx, ny, nz, 3), self.dtype)
        T = np.zeros((nx, ny, nz), self.dtype)
        rho0 = u0 = T0 = None
        if init_fields is not None:
            rho0, u0, T0 = (None if a is None else np.ascontiguousarray(a, dtype=self.dtype) for a in init_fields)
        ints = np.zeros(3, np.int32)
        dbl = np.zeros(4, np.float64)
        fn = self._fn("run_simulation")
        fn.restype = C.c_int
        D = C.c_double
        rc = fn(_p(mask), _p(hs), nx, ny, nz, int(max_steps), D(tau_fluid), D(heat_power), D(t_inlet),
                D(u_inlet_val), int(stats_every), D(tol_ke), D(tol_T), 1 if pump_mode == "constant_power" else 0,
                D(target_power), D(Pr), D(k_ratio), None if rho0 is None else _p(rho0),
                None if u0 is None else _p(u0), None if T0 is None else _p(T0), _p(rho), _p(u), _p(T), _p(ints),
                _p(dbl))
        if rc != 0:
            raise MemoryError("oracle run_simulation: allocation failed")
        return {"u": u, "rho": rho, "T": T, "mask": mask, "steps": int(ints[0]), "d_ke": float(dbl[0]),
                "dT_conv": float(dbl[1]), "dQ_conv": float(dbl[2]), "converged": bool(ints[1]),
                "diverged": bool(ints[2]), "u_inlet_final": float(dbl[3])}


def set_threads(n: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(n)
