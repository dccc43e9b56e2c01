"""ctypes binding of libxac.so (declared in include/xac.h).

The library is the only compute path: if it is missing or fails to load, importing anything that needs
it raises, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("XAC_LIB", _PKG / "libxac.so"))

XAC_OK, XAC_EINVAL, XAC_ECUDA, XAC_EDIVERGED, XAC_ETIMEOUT, XAC_ENOMEM = range(6)
BC_FLUID, BC_SOLID, BC_INLET, BC_OUTLET = 0, 1, 2, 3
FP32, FP16, BF16, FP32_T16 = 0, 1, 2, 3
# population storage: fp32 both lattices; fp16 both lattices; bf16 fluid with FP16 thermal; fp32_t16 FP32 fluid
# with FP16 thermal (include/xac.h gives their measured accuracy)
PRECISIONS = {"fp32": FP32, "fp16": FP16, "bf16": BF16, "fp32_t16": FP32_T16}

# stats slots (XAC_ST_*)
ST_MAX_V, ST_SUM_V, ST_SUM_KE, ST_COUNT, ST_SUM_RHO, ST_SUM_RHO_IN, ST_SUM_RHO_OUT, ST_SUM_UX_OUT = range(8)
ST_C_IN, ST_C_OUT, ST_C_OUTLET, ST_MAX_T, ST_SUM_T, ST_COUNT_T, ST_Q_OUT, ST_Q_OUT_COUNT, ST_NONFINITE = range(8, 17)
NSTATS = 17

SCALAR_NAMES = [
    "delta_P", "R_th", "Nu", "f_friction", "P_pump", "COP", "Q_vol", "T_max_surface", "T_avg_surface",
    "delta_T_max", "sigma_T", "fluid_temp_rise", "pressure_drop", "max_velocity", "max_temperature",
    "mean_temperature", "Dh", "V_fluid", "A_wetted", "porosity", "Q_absorbed", "dT_conv", "rho_avg",
]
NSCALARS = len(SCALAR_NAMES)

# validator slots (XAC_VAL_*)
VALIDATE_NAMES = ["mdot_in", "mdot_out", "max_v", "rho_dev", "T_min", "n_fluid", "rho1_all", "rho2_all", "div_sum",
                  "div_max", "div_n", "q_src", "adv_in", "adv_out", "diff_in", "diff_out"]
NVALIDATE = len(VALIDATE_NAMES)


class XacError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libxac error {code}: {msg}")
        self.code = code


class Desc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("mask", C.c_void_p), ("heat_source", C.c_void_p),
        ("tau_fluid", C.c_double), ("Pr", C.c_double), ("k_ratio", C.c_double),
        ("u_inlet", C.c_double), ("rho_outlet", C.c_double), ("t_inlet", C.c_double),
        ("heat_power", C.c_double), ("precision", C.c_int),
    ]


class ScalarParams(C.Structure):
    _fields_ = [
        ("buf", C.c_int), ("core_nx", C.c_int), ("core_ny", C.c_int),
        ("t_inlet", C.c_double), ("tau_fluid", C.c_double), ("Pr", C.c_double), ("u_inlet", C.c_double),
    ]


class RunOpts(C.Structure):
    _fields_ = [
        ("max_steps", C.c_int), ("stats_every", C.c_int), ("tol_ke", C.c_double), ("tol_T", C.c_double),
        ("constant_power", C.c_int), ("target_power", C.c_double), ("min_steps", C.c_int),
    ]


class DesignSpec(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("buf", C.c_int), ("family", C.c_int),
        ("margin", C.c_int), ("p0", C.c_double), ("p1", C.c_double), ("n_hot", C.c_int),
        ("background", C.c_double), ("hot", (C.c_double * 4) * 8),
    ]


DESIGN_FAMILIES = {"empty": 0, "straight": 1, "pin_fin": 2, "gyroid": 3, "schwarz_p": 4, "schwarz_d": 5}
DESIGN_BELOW = 16  # TPMS: solid where the value is below the threshold (generate_mask's convention)


class RunResult(C.Structure):
    _fields_ = [
        ("steps", C.c_longlong), ("converged", C.c_int), ("diverged", C.c_int),
        ("d_ke", C.c_double), ("dT_conv", C.c_double), ("dQ_conv", C.c_double),
        ("u_inlet_final", C.c_double), ("last_stats", C.c_double * NSTATS),
    ]


_vp, _i, _f, _d = C.c_void_p, C.c_int, C.c_float, C.c_double

# name -> argtypes (all return int)
SIGNATURES = {
    "xac_equilibrium": [_vp, _vp, _vp, _i, _i, _i, _vp],
    "xac_macroscopic": [_vp, _vp, _vp, _i, _i, _i, _vp],
    "xac_bgk_collision": [_vp, _vp, _vp, _vp, _f, _i, _i, _i, _vp],
    "xac_fused_collision": [_vp, _vp, _vp, _vp, _vp, _f, _i, _i, _i, _vp],
    "xac_stream": [_vp, _vp, _vp, _vp, _f, _i, _i, _i, _vp],
    "xac_stats_fields": [_vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp],
    "xac_stats_fields_noalloc": [_vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp],
    "xac_thermal_equilibrium": [_vp, _vp, _vp, _vp, _i, _i, _i, _vp],
    "xac_thermal_bgk_collision": [_vp, _vp, _vp, _vp, _f, _f, _vp, _f, _i, _i, _i, _vp],
    "xac_fused_thermal_collision": [_vp, _vp, _vp, _vp, _vp, _f, _f, _vp, _f, _i, _i, _i, _vp],
    "xac_thermal_stream": [_vp, _vp, _vp, _f, _i, _i, _i, _vp],
    "xac_thermal_macroscopic": [_vp, _vp, _i, _i, _i, _vp],
    "xac_test_dirichlet_plane": [_vp, _f, _i, _i, _i, _i, _vp],
    "xac_test_bounded_waits": [C.c_uint, _vp, _vp],
    "xac_test_set_step_status": [_vp, C.c_uint, _vp],
    "xac_test_conv_wait_timeout": [C.c_uint, _vp],
    "xac_test_periodic_stream": [_vp, _vp, _i, _i, _i, _vp],
    "xac_test_forced_bgk": [_vp, _vp, _vp, _vp, _f, _f, _i, _i, _i, _vp],
    "xac_test_periodic_stream_solids": [_vp, _vp, _vp, _i, _i, _i, _vp],
    "xac_test_couette_stream": [_vp, _vp, _vp, _f, _i, _i, _i, _vp],
    "xac_lattice_create": [C.POINTER(Desc), C.POINTER(_vp), _vp],
    "xac_reference_run_fp64": [C.POINTER(Desc), _i, _vp, _vp, _vp, _vp],
    "xac_lattice_destroy": [_vp],
    "xac_lattice_init_fields": [_vp, _vp, _vp, _vp, _vp],
    "xac_lattice_step": [_vp, _i, _vp],
    "xac_lattice_stats": [_vp, _vp, _vp],
    "xac_lattice_fields": [_vp, _vp, _vp, _vp, _vp],
    "xac_lattice_set_inlet": [_vp, _d, _vp],
    "xac_lattice_get_inlet": [_vp, C.POINTER(_d), _vp],
    "xac_lattice_steps_done": [_vp, C.POINTER(C.c_longlong)],
    "xac_lattice_tune": [_vp, _i, _i],
    "xac_lattice_pattern_copy": [_vp, _i, C.POINTER(_d), _vp],
    "xac_lattice_get_tune": [_vp, C.POINTER(_i), C.POINTER(_i)],
    "xac_lattice_scalars": [_vp, C.POINTER(ScalarParams), _vp, _vp],
    "xac_scalars_fields": [_vp, _vp, _vp, _vp, _i, _i, _i, C.POINTER(ScalarParams), _vp, _vp],
    "xac_lattice_state_bytes": [_vp, C.POINTER(C.c_size_t)],
    "xac_lattice_save_state": [_vp, _vp, C.c_size_t, _vp],
    "xac_lattice_load_state": [_vp, _vp, C.c_size_t, _vp],
    "xac_lattice_run": [_vp, C.POINTER(RunOpts), C.POINTER(RunResult), _vp],
    "xac_lattice_validate": [_vp, _vp, _vp],
    "xac_design_build": [C.POINTER(DesignSpec), _vp, _vp, _vp],
    "xac_conv3d_forward": [_vp, _i, _i, _i, _i, _i, _vp, _vp, _i, _i, _i, _vp, _vp, _vp],
    "xac_conv3d_weight_grad": [_vp, _i, _i, _i, _i, _i, _vp, _i, _i, _vp, _vp, _vp, _vp],
    "xac_conv3d_partial_floats": [_i, _i, _i, _i, _i, _i, _i, C.POINTER(C.c_longlong)],
    "xac_conv3d_status": [C.POINTER(_i)],
    "xac_batch_create": [C.POINTER(Desc), _i, C.POINTER(_vp), _vp],
    "xac_batch_destroy": [_vp],
    "xac_batch_size": [_vp, C.POINTER(_i)],
    "xac_batch_lattice": [_vp, _i, C.POINTER(_vp)],
    "xac_batch_tune": [_vp, _i, _i],
    "xac_batch_get_tune": [_vp, C.POINTER(_i), C.POINTER(_i)],
    "xac_batch_run": [_vp, C.POINTER(RunOpts), C.POINTER(RunResult), _vp],
    "xac_batch_launch_counts": [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "xac_batch_open": [_i, C.POINTER(_vp)],
    "xac_batch_admit": [_vp, C.POINTER(Desc), C.POINTER(_i), _vp],
    "xac_batch_advance": [_vp, C.POINTER(RunOpts), C.c_longlong, C.POINTER(_i), C.POINTER(_i), C.POINTER(RunResult),
                          C.POINTER(_d), _vp],
    "xac_batch_release": [_vp, _i],
    "xac_lattice_footprint": [C.POINTER(Desc), C.POINTER(C.c_ulonglong)],
}

_lib = None


def load() -> C.CDLL:
    """Load libxac.so once; raise with a clear message when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m xadvcool_b200.build` "
            "(there is no CPU fallback for the solver)"
        )
    lib = C.CDLL(str(LIB_PATH))
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = C.c_int
    lib.xac_last_error.argtypes = []
    lib.xac_last_error.restype = C.c_char_p
    lib.xac_version.argtypes = []
    lib.xac_version.restype = C.c_int
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != XAC_OK:
        msg = load().xac_last_error().decode(errors="replace")
        raise XacError(rc, msg)


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
