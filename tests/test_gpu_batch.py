"""The persistent batched solve against solo solves of the same designs: identical step counts, convergence
flags and fields (same kernels, same deterministic stats reduction)."""
import numpy as np
import pytest
import torch

from xadvcool_b200 import designs
from xadvcool_b200.batch import Batch
from xadvcool_b200.lattice import Lattice

pytestmark = pytest.mark.gpu


def small_designs():
    out = []
    for s, shape in enumerate([(40, 18, 10), (64, 24, 12), (52, 20, 9)]):
        m, hs, u, info = designs.gyroid_design(s, nx=shape[0], ny=shape[1], nz=shape[2], buf=4)
        out.append(dict(mask=m, heat_source=hs, tau_fluid=0.6 + 0.02 * s, u_inlet_val=min(u, 0.04), Pr=2.0,
                        k_ratio=20.0, heat_power=0.02))
    m = designs.straight_fin_plate()
    out.append(dict(mask=m, tau_fluid=0.6, heat_power=1e-4, u_inlet_val=0.05, Pr=2.0, k_ratio=100.0))
    return out


def solo(d, **run):
    lat = Lattice(d["mask"], **{k: v for k, v in d.items() if k != "mask"})
    res = lat.run(**run)
    f = [t.cpu().numpy() for t in lat.fields()]
    lat.close()
    return res, f


@pytest.mark.parametrize("block,spl", [(128, 1000), (64, 250), (256, 7)])
def test_batch_equals_solo_solves(block, spl, cuda):
    ds = small_designs()
    run = dict(max_steps=9000, stats_every=100, tol_ke=2e-4, tol_T=2e-4)
    b = Batch(ds)
    b.tune(block, spl)
    res = b.run(**run)
    for i, d in enumerate(ds):
        ref, f_ref = solo(d, **run)
        assert res[i]["steps"] == ref["steps"], (i, res[i]["steps"], ref["steps"])
        assert res[i]["converged"] == ref["converged"] and res[i]["diverged"] == ref["diverged"]
        assert res[i]["d_ke"] == ref["d_ke"]
        f = [t.cpu().numpy() for t in b.lattice(i).fields()]
        for a, c in zip(f, f_ref):
            assert np.array_equal(a, c)
    assert len({r["steps"] for r in res}) > 1  # designs retired at different steps


def test_batch_divergence_retires_only_the_diverging_design(cuda):
    ds = small_designs()[:2]
    ds[1] = dict(ds[1], u_inlet_val=0.3, tau_fluid=0.51)
    b = Batch(ds)
    res = b.run(max_steps=3000, stats_every=100, tol_ke=0.0, tol_T=0.0)
    assert res[1]["diverged"] and not res[0]["diverged"]
    assert res[0]["steps"] == 3000 and res[1]["steps"] < 3000


def test_batch_warm_start_and_fp16(cuda):
    ds = small_designs()[:2]
    b = Batch(ds, precision="fp16")
    lat0 = b.lattice(0)
    rho, u, T = lat0.fields()
    lat0.init_fields(rho, u, T + 1.0)
    res = b.run(max_steps=500, stats_every=100, tol_ke=0.0, tol_T=0.0)
    assert all(r["steps"] == 500 for r in res)
    s0 = b.lattice(0).stats()
    assert np.isfinite(s0).all() and s0[16] == 0


def test_batch_rejects_bad_input(cuda):
    ds = small_designs()[:1]
    b = Batch(ds)
    with pytest.raises(Exception):
        b.tune(100, 10)
    b.run(max_steps=200, stats_every=100)
    with pytest.raises(Exception):  # designs must restart from step 0
        b.run(max_steps=200, stats_every=100)


@pytest.mark.parametrize("spl", [1000, 300])
def test_batch_constant_power_equals_solo(spl, cuda):
    """The pump controller inside the persistent kernel (src/simulation.py:139-146) gives each design the inlet
    history, step count and fields of its solo constant-power solve, bit for bit."""
    ds = small_designs()[:3]
    run = dict(max_steps=3000, stats_every=100, tol_ke=1e-6, tol_T=1e-6, pump_mode="constant_power",
               target_power=0.02)
    b = Batch(ds)
    b.tune(128, spl)
    res = b.run(**run)
    for i, d in enumerate(ds):
        r_solo, f_solo = solo(d, **run)
        assert res[i]["steps"] == r_solo["steps"]
        assert res[i]["u_inlet_final"] == r_solo["u_inlet_final"]
        assert res[i]["u_inlet_final"] != pytest.approx(d["u_inlet_val"], rel=1e-3)  # the pump acted
        lat = b.lattice(i)
        assert lat.get_inlet() == pytest.approx(r_solo["u_inlet_final"], rel=0, abs=0)
        for x, y in zip([t.cpu().numpy() for t in lat.fields()], f_solo):
            assert np.array_equal(x, y)
    b.close()


def test_batch_tile_autotune(cuda, tmp_path, monkeypatch):
    """The batch autotuner times every tile on scratch batches, caches the winner, and sets it; the tuned batch
    still solves exactly as the solo lattices do."""
    from xadvcool_b200 import autotune
    monkeypatch.setenv("XAC_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    ds = small_designs()
    res = autotune.autotune_batch(ds, steps=200)
    assert res["block"] in autotune.BATCH_BLOCKS
    assert sorted(res["table"]) == sorted(str(b) for b in autotune.BATCH_BLOCKS)
    assert autotune.autotune_batch(ds, steps=200) == res  # cached
    b = Batch(ds)
    autotune.apply_batch(b, ds, steps=200)
    assert b.get_tune()[0] == res["block"]
    run = dict(max_steps=600, stats_every=100, tol_ke=0.0, tol_T=0.0)
    out = b.run(**run)
    for i, d in enumerate(ds):
        ref, f_ref = solo(d, **run)
        assert out[i]["steps"] == ref["steps"] and out[i]["d_ke"] == ref["d_ke"]
        for a, c in zip((t.cpu().numpy() for t in b.lattice(i).fields()), f_ref):
            assert np.array_equal(a, c)
    b.close()


C4_SEEDS = (0, 1, 2, 4, 6, 7, 9, 10, 18)  # every x in {96,128,148,192}, y in {64,96,128}, z in {16,32,48}, 5 families


def c4_designs():
    out = []
    for s in C4_SEEDS:
        m, hs, u, info = designs.mixed_design(s)
        out.append(dict(mask=m, heat_source=hs, tau_fluid=0.56, u_inlet_val=u, Pr=7.0, k_ratio=628.0,
                        heat_power=0.1))
    out[7] = dict(out[7], u_inlet_val=0.3, tau_fluid=0.51)  # 148x64x16 straight channel: retires by divergence
    return out


def test_batch_of_dataset_shapes_equals_solo_solves(cuda):
    """Nine designs of the batching workload's shapes and families (up to 192x96x32 and 148x96x48, 3.3 M cells) in
    one persistent launch, retiring at different steps by convergence or divergence: each design's step count,
    flags, convergence rates and fields equal its solo solve bit for bit."""
    ds = c4_designs()
    run = dict(max_steps=2000, stats_every=100, tol_ke=1e-3, tol_T=1e-3, min_steps=200)
    b = Batch(ds)
    res = b.run(**run)
    steps = [r["steps"] for r in res]
    print("batch steps:", steps)
    for i, d in enumerate(ds):
        ref, f_ref = solo(d, **run)
        assert res[i]["steps"] == ref["steps"], (i, res[i]["steps"], ref["steps"])
        assert res[i]["converged"] == ref["converged"] and res[i]["diverged"] == ref["diverged"]
        assert res[i]["d_ke"] == ref["d_ke"] and res[i]["dQ_conv"] == ref["dQ_conv"]
        for a, c in zip((t.cpu().numpy() for t in b.lattice(i).fields()), f_ref):
            assert np.array_equal(a.view(np.uint32), c.view(np.uint32))  # bit patterns: the diverged one holds NaN
    assert res[7]["diverged"] and any(r["converged"] for r in res)
    assert len(set(steps)) >= 3  # retirement interleaves
    b.close()


@pytest.mark.parametrize("precision", ["fp32_t16", "bf16"])
def test_batch_equals_solo_with_reduced_storage(precision, cuda):
    """The persistent batch kernel with FP32 fluid / scaled FP16 thermal storage and with BF16 fluid storage: step
    counts and fields equal the solo solves bit for bit."""
    ds = small_designs()[:3]
    run = dict(max_steps=1500, stats_every=100, tol_ke=2e-4, tol_T=2e-4)
    with Batch(ds, precision=precision) as b:
        res = b.run(**run)
        got = [[t.cpu().numpy() for t in b.lattice(i).fields()] for i in range(len(ds))]
    for i, d in enumerate(ds):
        with Lattice(d["mask"], precision=precision, **{k: v for k, v in d.items() if k != "mask"}) as lat:
            ref = lat.run(**run)
            want = [t.cpu().numpy() for t in lat.fields()]
        assert res[i]["steps"] == ref["steps"] and res[i]["converged"] == ref["converged"]
        for a, c in zip(got[i], want):
            assert np.array_equal(a, c)
