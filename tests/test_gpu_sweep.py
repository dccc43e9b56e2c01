"""Open batches (designs joining and leaving a running persistent batch) and the sweep queue built on them, against
solo solves: every design keeps the step count, flags, convergence rates, fields and scalars of its own
xac_lattice_run, bit for bit, whenever it joins."""
import numpy as np
import pytest

from xadvcool_b200 import designs, sweep
from xadvcool_b200.batch import Batch, footprint
from xadvcool_b200.lattice import Lattice

pytestmark = pytest.mark.gpu

RUN = dict(max_steps=2500, stats_every=100, tol_ke=1e-3, tol_T=1e-3, min_steps=300)


def queue_designs():
    out = []
    for s, shape in enumerate([(64, 24, 12), (40, 18, 10), (96, 32, 16), (52, 20, 9), (72, 28, 14), (48, 16, 8)]):
        m, hs, u, _ = designs.gyroid_design(s, nx=shape[0], ny=shape[1], nz=shape[2], buf=4)
        out.append(dict(mask=m, heat_source=hs, tau_fluid=0.58 + 0.01 * s, u_inlet_val=min(u, 0.04), Pr=3.0,
                        k_ratio=30.0, heat_power=0.02))
    out[3] = dict(out[3], u_inlet_val=0.3, tau_fluid=0.51)  # diverges
    return out


def solo(d, **run):
    lat = Lattice(d["mask"], **{k: v for k, v in d.items() if k != "mask"})
    res = lat.run(**run)
    f = [t.cpu().numpy() for t in lat.fields()]
    sc = lat.scalars(buf=4, core_nx=d["mask"].shape[0] - 8, core_ny=d["mask"].shape[1])
    lat.close()
    return res, f, sc


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def test_open_batch_designs_joining_mid_run_equal_solo_solves(cuda):
    """Two designs start the batch; the others join one at a time as slots free up, at whatever step the batch
    has reached (launches of 250 steps, so a design admitted between launches waits for the next stats boundary)."""
    ds = queue_designs()
    with Batch.open() as b:
        b.tune(128, 250)
        live = {b.admit(ds[0]): 0, b.admit(ds[1]): 1}
        queue = list(range(2, len(ds)))
        got = {}
        while live:
            for f in b.advance(650, **RUN):
                i = live.pop(f["slot"])
                lat = b.lattice(f["slot"])
                got[i] = (f, [t.cpu().numpy() for t in lat.fields()],
                          lat.scalars(buf=4, core_nx=ds[i]["mask"].shape[0] - 8, core_ny=ds[i]["mask"].shape[1]))
                b.release(f["slot"])
                if queue:
                    j = queue.pop(0)
                    live[b.admit(ds[j])] = j
        assert len(b) <= 3  # released slots are reused
        graphs, direct = b.launch_counts()
        assert graphs > 0
    assert sorted(got) == list(range(len(ds)))
    for i, d in enumerate(ds):
        ref, f_ref, sc_ref = solo(d, **RUN)
        f, fields, sc = got[i]
        assert f["steps"] == ref["steps"], (i, f["steps"], ref["steps"])
        assert f["converged"] == ref["converged"] and f["diverged"] == ref["diverged"]
        assert f["d_ke"] == ref["d_ke"] and f["dQ_conv"] == ref["dQ_conv"]
        assert f["gpu_seconds"] > 0
        for a, c in zip(fields, f_ref):
            assert same_bits(a, c)
        if not ref["diverged"]:
            assert sc["delta_P"] == sc_ref["delta_P"] and sc["R_th"] == sc_ref["R_th"]
    assert got[3][0]["diverged"] and any(g[0]["converged"] for g in got.values())


def test_sweep_queue_under_a_two_design_budget_equals_solo_solves(cuda):
    ds = [d for k, d in enumerate(queue_designs()) if k != 3]
    budget = 2 * max(footprint(d) for d in ds)
    rows = sweep.solve_shard(ds, list(range(len(ds))), max_steps=2500, tol=1e-3, budget_bytes=budget, buf=4,
                             core=(32, 16), steps_per_launch=200)
    assert sorted(rows[:, 0].astype(int)) == list(range(len(ds)))
    for r in rows:
        d = ds[int(r[0])]
        lat = Lattice(d["mask"], **{k: v for k, v in d.items() if k != "mask"})
        ref = lat.run(max_steps=2500, stats_every=100, tol_ke=1e-3, tol_T=1e-3)
        sc = lat.scalars(buf=4, core_nx=32, core_ny=16)
        lat.close()
        assert r[1] == ref["steps"] and bool(r[2]) == ref["converged"] and bool(r[3]) == ref["diverged"]
        assert r[4] == sc["delta_P"] and r[5] == sc["R_th"] and r[6] == sc["Nu"]
        assert r[11] > 0 and r[12] > 0


def test_closed_batch_runs_from_a_captured_graph(cuda):
    """The persistent launches of xac_batch_run replay a captured CUDA graph (the driver allows capturing the
    cooperative launch here); a direct launch would show in the counts."""
    ds = queue_designs()[:2]
    with Batch(ds) as b:
        b.run(max_steps=400, stats_every=100, tol_ke=0.0, tol_T=0.0)
        graphs, direct = b.launch_counts()
    assert graphs >= 1 and direct == 0


def test_open_batch_rejects_misuse(cuda):
    ds = queue_designs()
    with Batch.open() as b:
        with pytest.raises(Exception):
            b.run(max_steps=100)  # an open batch advances, it does not run
        k = b.admit(ds[0])
        with pytest.raises(Exception):
            b.release(k + 1)  # empty slot
        b.advance(100, **RUN)
        with pytest.raises(Exception):
            b.release(k)  # still running
