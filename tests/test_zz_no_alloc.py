"""xac_stats_fields_noalloc, the stats entry point for callers that cannot allocate memory (code inside a
stream capture, or running under a memory budget owned by another allocator): checked through the C ABI
against xac_stats_fields on the same fields, on two calls in a row. This file is collected last on purpose,
so a run that stops at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

from xadvcool_b200 import _capi

pytestmark = pytest.mark.gpu


def _fields(seed, shape, dev):
    rng = np.random.default_rng(seed)
    mask = rng.choice([0, 0, 0, 1, 1, 2, 3], size=shape).astype(np.int32)
    rho = rng.uniform(0.95, 1.05, size=shape).astype(np.float32)
    u = rng.uniform(-0.08, 0.08, size=shape + (3,)).astype(np.float32)
    T = rng.uniform(20.0, 60.0, size=shape).astype(np.float32)
    return [torch.from_numpy(a).to(dev) for a in (rho, u, T, mask)]


def test_no_alloc_stats_equal_the_allocating_entry_point_on_two_calls(cuda):
    lib = _capi.load()
    stream = torch.cuda.current_stream(cuda).cuda_stream
    # the larger lattice first, so the second call runs over scratch rows left by the first
    for seed, shape in ((11, (148, 128, 32)), (12, (37, 19, 23))):
        rho, u, T, mask = _fields(seed, shape, cuda)
        ptrs = (rho.data_ptr(), u.data_ptr(), T.data_ptr(), mask.data_ptr())
        ref = np.zeros(_capi.NSTATS, dtype=np.float64)
        _capi.check(lib.xac_stats_fields(*ptrs, *shape, ref.ctypes.data, stream))
        out = torch.full((_capi.NSTATS,), float("nan"), dtype=torch.float64, device=cuda)
        _capi.check(lib.xac_stats_fields_noalloc(*ptrs, *shape, out.data_ptr(), stream))
        torch.cuda.synchronize(cuda)
        np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-12, atol=1e-12)


def test_no_alloc_rejects_lattices_beyond_its_scratch(cuda):
    lib = _capi.load()
    dummy = torch.zeros(16, dtype=torch.float32, device=cuda)
    out = torch.zeros(_capi.NSTATS, dtype=torch.float64, device=cuda)
    p = dummy.data_ptr()
    rc = lib.xac_stats_fields_noalloc(p, p, p, p, 2048, 1025, 1, out.data_ptr(), None)
    assert rc == _capi.XAC_EINVAL
    assert b"exceed the fixed scratch" in lib.xac_last_error()
