"""Each unfused CUDA operator (reference layout) against the C oracle on the same seeded inputs:
bit-exact (both sides round every multiply and add separately, in the reference's operand order)."""
import numpy as np
import pytest
import torch

from gpu_backend import GpuBackend
from oracle.ref import Ref

pytestmark = pytest.mark.gpu

SHAPES = [(7, 5, 6), (16, 9, 12), (33, 17, 8)]


def rand_case(shape, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    m = rng.choice([0, 0, 0, 1, 2, 3], size=shape).astype(np.int32)
    f = (rng.uniform(0.005, 0.12, size=(19,) + shape)).astype(np.float32)
    rho = rng.uniform(0.9, 1.1, size=shape).astype(np.float32)
    u = rng.uniform(-0.06, 0.06, size=shape + (3,)).astype(np.float32)
    T = rng.uniform(20.0, 45.0, size=shape).astype(np.float32)
    hs = np.where(rng.random(shape) < 0.3, rng.random(shape), 0.0).astype(np.float32)
    return m, f, rho, u, T, hs


def gpu(a):
    return GpuBackend().array(a)


@pytest.fixture(scope="module")
def ref():
    return Ref(32)


@pytest.mark.parametrize("shape", SHAPES)
def test_equilibrium_and_macroscopic(shape, ref, cuda):
    m, f, rho, u, T, hs = rand_case(shape, 1)
    be = GpuBackend()
    out_c, out_g = np.zeros((19,) + shape, np.float32), be.zeros((19,) + shape)
    ref.compute_equilibrium_kernel(rho, u, out_c)
    be.compute_equilibrium_kernel(gpu(rho), gpu(u), out_g)
    assert np.array_equal(out_c, be.numpy(out_g))
    r_c, u_c = np.zeros(shape, np.float32), np.zeros(shape + (3,), np.float32)
    r_g, u_g = be.zeros(shape), be.zeros(shape + (3,))
    ref.compute_macroscopic_kernel(f, r_c, u_c)
    be.compute_macroscopic_kernel(gpu(f), r_g, u_g)
    assert np.array_equal(r_c, be.numpy(r_g)) and np.array_equal(u_c, be.numpy(u_g))


@pytest.mark.parametrize("shape", SHAPES)
def test_collisions(shape, ref, cuda):
    m, f, rho, u, T, hs = rand_case(shape, 2)
    be = GpuBackend()
    feq = np.zeros_like(f)
    ref.compute_equilibrium_kernel(rho, u, feq)
    a_c, a_g = np.zeros_like(f), be.zeros(f.shape)
    ref.bgk_collision_kernel(f, feq, a_c, m, 0.57)
    be.bgk_collision_kernel(gpu(f), gpu(feq), a_g, gpu(m), 0.57)
    assert np.array_equal(a_c, be.numpy(a_g))
    ref.fused_equilibrium_collision_kernel(f, rho, u, a_c, m, 0.53)
    be.fused_equilibrium_collision_kernel(gpu(f), gpu(rho), gpu(u), a_g, gpu(m), 0.53)
    assert np.array_equal(a_c, be.numpy(a_g))
    ref.fused_thermal_equilibrium_collision_kernel(f, u, T, a_c, m, 0.507, 4.99, hs, 0.13)
    be.fused_thermal_equilibrium_collision_kernel(gpu(f), gpu(u), gpu(T), a_g, gpu(m), 0.507, 4.99, gpu(hs), 0.13)
    assert np.array_equal(a_c, be.numpy(a_g))
    geq = np.zeros_like(f)
    ref.compute_thermal_equilibrium_kernel(rho, u, T, geq, m)
    g_g = be.zeros(f.shape)
    be.compute_thermal_equilibrium_kernel(gpu(rho), gpu(u), gpu(T), g_g, gpu(m))
    assert np.array_equal(geq, be.numpy(g_g))
    ref.thermal_bgk_collision_kernel(f, geq, a_c, m, 0.55, 5.5, hs, 1e-3)
    be.thermal_bgk_collision_kernel(gpu(f), g_g, a_g, gpu(m), 0.55, 5.5, gpu(hs), 1e-3)
    assert np.array_equal(a_c, be.numpy(a_g))


@pytest.mark.parametrize("shape", SHAPES)
def test_streaming_operators(shape, ref, cuda):
    m, f, rho, u, T, hs = rand_case(shape, 3)
    be = GpuBackend()
    nx, ny, nz = shape
    pre = np.random.default_rng(9).random((19,) + shape).astype(np.float32)  # solid cells keep these
    s_c, s_g = pre.copy(), gpu(pre)
    ref.streaming_kernel(f, s_c, m, np.array([0.043], np.float32), 1.0, nx, ny, nz)
    be.streaming_kernel(gpu(f), s_g, gpu(m), gpu(np.array([0.043], np.float32)), 1.0, nx, ny, nz)
    assert np.array_equal(s_c, be.numpy(s_g))
    t_c, t_g = np.zeros_like(f), be.zeros(f.shape)
    ref.thermal_streaming_kernel(f, t_c, m, 25.0, nx, ny, nz)
    be.thermal_streaming_kernel(gpu(f), t_g, gpu(m), 25.0, nx, ny, nz)
    assert np.array_equal(t_c, be.numpy(t_g))
    T_c, T_g = np.zeros(shape, np.float32), be.zeros(shape)
    ref.compute_thermal_macroscopic_kernel(f, T_c)
    be.compute_thermal_macroscopic_kernel(gpu(f), T_g)
    assert np.array_equal(T_c, be.numpy(T_g))


@pytest.mark.parametrize("shape", SHAPES)
def test_test_only_operators(shape, ref, cuda):
    m, f, rho, u, T, hs = rand_case(shape, 4)
    m = np.where(m > 1, 0, m).astype(np.int32)
    be = GpuBackend()
    nx, ny, nz = shape
    pre = np.random.default_rng(8).random((19,) + shape).astype(np.float32)
    for name, args in (("periodic_streaming_kernel", (nx, ny, nz)),
                       ("periodic_streaming_with_solids_kernel", ("M", nx, ny, nz)),
                       ("couette_streaming_kernel", ("M", 0.05, nx, ny, nz))):
        c, g = pre.copy(), gpu(pre)
        getattr(ref, name)(f, c, *[m if a == "M" else a for a in args])
        getattr(be, name)(gpu(f), g, *[gpu(m) if a == "M" else a for a in args])
        assert np.array_equal(c, be.numpy(g)), name
    feq = np.zeros_like(f)
    ref.compute_equilibrium_kernel(rho, u, feq)
    c, g = np.zeros_like(f), be.zeros(f.shape)
    ref.forced_bgk_collision_kernel(f, feq, c, m, 0.8, 1e-5)
    be.forced_bgk_collision_kernel(gpu(f), gpu(feq), g, gpu(m), 0.8, 1e-5)
    assert np.array_equal(c, be.numpy(g))
    c, g = f.copy(), gpu(f)
    ref.dirichlet_thermal_bc_kernel(c, 100.0, 0, ny, nz)
    be.dirichlet_thermal_bc_kernel(g, 100.0, 0, ny, nz)
    assert np.array_equal(c, be.numpy(g))


def test_field_stats_match_oracle(ref, cuda):
    from xadvcool_b200.fluid_engine3d import field_stats
    m, f, rho, u, T, hs = rand_case((20, 11, 9), 5)
    s_c = ref.stats(rho, u, T, m)
    s_g = field_stats(gpu(rho), gpu(u), gpu(T), gpu(m))
    assert np.allclose(s_c, s_g, rtol=1e-12, atol=1e-12)


def test_bad_arguments_raise(cuda):
    from xadvcool_b200 import fluid_engine3d as fe
    be = GpuBackend()
    with pytest.raises(TypeError):
        fe.compute_equilibrium_kernel(be.zeros((3, 3, 3)).double(), be.zeros((3, 3, 3, 3)), be.zeros((19, 3, 3, 3)))
    with pytest.raises(ValueError):
        fe.compute_equilibrium_kernel(torch.zeros(3, 3, 3), be.zeros((3, 3, 3, 3)), be.zeros((19, 3, 3, 3)))
