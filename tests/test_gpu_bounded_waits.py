"""Failure detection without a GPU fault: the library's bounded waits (the staged step kernel's mbarrier wait,
the batched kernel's grid barrier) are made to run out on purpose, through a test-only entry point, with a wait
that nothing completes. Each must give up after its limit and report, and the context must stay usable."""
import ctypes as C

import numpy as np
import pytest
import torch

from xadvcool_b200 import _capi, designs
from xadvcool_b200._tensors import stream_ptr
from xadvcool_b200.lattice import Lattice

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("limit", [1, 1000])
def test_bounded_waits_give_up_and_report(limit, cuda):
    st = C.c_uint(0)
    _capi.call("xac_test_bounded_waits", limit, C.byref(st), stream_ptr(torch.device("cuda")))
    assert st.value == 7  # mbarrier wait gave up, grid barrier gave up and recorded XAC_ETIMEOUT
    # the context is still usable: a solve right after runs, on the staged kernel, with finite stats
    mask = designs.straight_fin_plate()
    with Lattice(mask, tau_fluid=0.6, heat_power=1e-4, u_inlet_val=0.05, Pr=2.0, k_ratio=100.0) as lat:
        lat.tune(128, 1)  # the staged kernel, whose wait is the one exercised above
        lat.step(20)
        s = lat.stats()
    assert np.isfinite(s).all() and s[16] == 0


def test_bounded_waits_reject_bad_limit(cuda):
    st = C.c_uint(0)
    with pytest.raises(_capi.XacError):
        _capi.call("xac_test_bounded_waits", 0, C.byref(st), None)


def test_conv_wait_gives_up_and_reports(cuda):
    from xadvcool_b200 import surrogate as S
    S.kernel_status()  # clears the flags
    _capi.call("xac_test_conv_wait_timeout", 1000, stream_ptr(torch.device("cuda")))
    assert S.kernel_status() & 1
    assert S.kernel_status() == 0  # read-and-clear


def test_staged_wait_failure_is_fatal_until_the_populations_are_rewritten(cuda):
    """After the staged kernel's status word reports a wait that gave up (written here by a test hook, as the kernel
    would), the lattice refuses steps, runs, stats, fields and scalars with XAC_ETIMEOUT; init_fields rewrites
    every population and makes it usable again, and the solve from there matches a fresh lattice."""
    mask = designs.straight_fin_plate()
    kw = dict(tau_fluid=0.6, heat_power=1e-4, u_inlet_val=0.05, Pr=2.0, k_ratio=100.0)
    dev = torch.device("cuda")
    with Lattice(mask, **kw) as lat:
        lat.tune(128, 1)
        lat.step(10)
        _capi.call("xac_test_set_step_status", lat._h, 1, stream_ptr(dev))
        with pytest.raises(_capi.XacError) as e:
            lat.stats()
        assert e.value.code == _capi.XAC_ETIMEOUT
        for call in (lambda: lat.step(1), lat.stats, lat.fields, lambda: lat.scalars(buf=8, core_nx=48, core_ny=32),
                     lambda: lat.run(max_steps=200)):
            with pytest.raises(_capi.XacError) as e:
                call()
            assert e.value.code == _capi.XAC_ETIMEOUT and "init_fields" in str(e.value)
        lat.init_fields()  # cold start again
        lat.step(30)
        got = [t.cpu().numpy() for t in lat.fields()]
    with Lattice(mask, **kw) as ref:
        ref.step(30)
        want = [t.cpu().numpy() for t in ref.fields()]
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
