"""xadvcool_b200 — B200-native coupled fluid + thermal lattice-Boltzmann solver behind the
fluid_engine3d / thermal_engine3d / simulation API of tgautam03/xAdvCool.

The compute path is libxac.so (hand-written sm_100a kernels, C ABI in include/xac.h); it must be built
(``python -m xadvcool_b200.build``) and there is no CPU fallback.
"""
from . import _capi  # noqa: F401

__version__ = "0.1.0"


def lib():
    """Load libxac.so (raises if it has not been built)."""
    return _capi.load()
