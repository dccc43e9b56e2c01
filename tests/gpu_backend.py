"""Backend for tests/analytical_cases.py on libxac.so's CUDA operators (torch CUDA tensors), including the
test-only kernels of validate_analytical.py that libxac.so exports as xac_test_*."""
from __future__ import annotations

import numpy as np
import torch

from xadvcool_b200 import _capi, fluid_engine3d as fe, thermal_engine3d as te
from xadvcool_b200._tensors import dev_ptr, stream_ptr

F32, I32 = torch.float32, torch.int32


class GpuBackend:
    def __init__(self, device="cuda:0"):
        self.dev = torch.device(device)

    def zeros(self, shape):
        return torch.zeros(shape, dtype=F32, device=self.dev)

    def full(self, shape, v):
        return torch.full(shape, float(v), dtype=F32, device=self.dev)

    def array(self, a):
        a = np.asarray(a)
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.to(self.dev, dtype=I32 if a.dtype == np.int32 else F32)

    def numpy(self, t):
        return t.cpu().numpy()

    def copy(self, dst, src):
        dst.copy_(src)

    # product operators (reference names)
    compute_equilibrium_kernel = staticmethod(fe.compute_equilibrium_kernel)
    compute_macroscopic_kernel = staticmethod(fe.compute_macroscopic_kernel)
    bgk_collision_kernel = staticmethod(fe.bgk_collision_kernel)
    fused_equilibrium_collision_kernel = staticmethod(fe.fused_equilibrium_collision_kernel)
    streaming_kernel = staticmethod(fe.streaming_kernel)
    compute_thermal_equilibrium_kernel = staticmethod(te.compute_thermal_equilibrium_kernel)
    thermal_bgk_collision_kernel = staticmethod(te.thermal_bgk_collision_kernel)
    fused_thermal_equilibrium_collision_kernel = staticmethod(te.fused_thermal_equilibrium_collision_kernel)
    thermal_streaming_kernel = staticmethod(te.thermal_streaming_kernel)
    compute_thermal_macroscopic_kernel = staticmethod(te.compute_thermal_macroscopic_kernel)

    # test-only operators
    @staticmethod
    def dirichlet_thermal_bc_kernel(g, T_val, x_plane, ny, nz):
        nx = g.shape[1]
        _capi.call("xac_test_dirichlet_plane", dev_ptr(g, F32, "g"), float(T_val), int(x_plane), nx, ny, nz,
                   stream_ptr())

    @staticmethod
    def periodic_streaming_kernel(fp, fs, nx, ny, nz):
        _capi.call("xac_test_periodic_stream", dev_ptr(fp, F32, "fp"), dev_ptr(fs, F32, "fs"), nx, ny, nz,
                   stream_ptr())

    periodic_thermal_streaming_kernel = periodic_streaming_kernel

    @staticmethod
    def forced_bgk_collision_kernel(f_old, f_eq, f_new, mask, tau, force_x):
        _, nx, ny, nz = f_old.shape
        _capi.call("xac_test_forced_bgk", dev_ptr(f_old, F32, "f_old"), dev_ptr(f_eq, F32, "f_eq"),
                   dev_ptr(f_new, F32, "f_new"), dev_ptr(mask, I32, "mask"), float(tau), float(force_x), nx, ny, nz,
                   stream_ptr())

    @staticmethod
    def periodic_streaming_with_solids_kernel(fp, fs, mask, nx, ny, nz):
        _capi.call("xac_test_periodic_stream_solids", dev_ptr(fp, F32, "fp"), dev_ptr(fs, F32, "fs"),
                   dev_ptr(mask, I32, "mask"), nx, ny, nz, stream_ptr())

    @staticmethod
    def couette_streaming_kernel(fp, fs, mask, u_wall_x, nx, ny, nz):
        _capi.call("xac_test_couette_stream", dev_ptr(fp, F32, "fp"), dev_ptr(fs, F32, "fs"),
                   dev_ptr(mask, I32, "mask"), float(u_wall_x), nx, ny, nz, stream_ptr())
