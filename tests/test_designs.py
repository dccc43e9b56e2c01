"""Design generator vs the reference's generate_mask / heat maps (hashes in tests/golden/designs.json,
made by tests/golden/make_golden.py from src/geometry.py) and vs the dataset's porosity / Dh."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from xadvcool_b200 import designs, metrics

GOLD = Path(__file__).resolve().parent / "golden"
D = json.loads((GOLD / "designs.json").read_text())
ROWS = json.loads((GOLD / "parquet_rows.json").read_text())


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", D["masks"], ids=lambda c: "t{design_type}-{feature_size}-{spacing}".format(**c["state"]))
def test_generate_mask_matches_reference(case):
    m = designs.generate_mask(case["state"])
    assert list(m.shape) == case["shape"]
    assert sha(m.astype(np.int32)) == case["sha256"]


@pytest.mark.parametrize("key", sorted(D["heat_maps"]))
def test_heat_maps_match_reference(key):
    name, seed = key.split(":")
    hm = designs.HEAT_SOURCE_REGISTRY[name](128, 128, seed=int(seed)).astype(np.float32)
    g = D["heat_maps"][key]
    if sha(hm) != g["sha256"]:  # blur results may differ in the last bit across scipy builds
        assert abs(float(hm.astype(np.float64).sum()) - g["sum"]) < 1e-4 * max(1.0, g["sum"])
        assert np.allclose([hm[17, 33], hm[64, 64], hm[101, 90]], g["probe"], rtol=1e-6, atol=1e-7)
    assert float(hm.max()) == g["max"]


@pytest.mark.parametrize("row", ROWS, ids=lambda r: r["sample_id"])
def test_dataset_row_geometry(row):
    state = {"design_type": row["design_idx"], "feature_size": row["feature_size"], "spacing": row["spacing"],
             "buffer_size": 10}
    m = designs.generate_mask(state)
    assert sha(m.astype(np.int32)) == row["mask_sha256"]
    Dh, V, A = metrics.compute_hydraulic_diameter(m)
    assert Dh == pytest.approx(row["Dh"], rel=1e-12)
    assert metrics.compute_porosity(m) == pytest.approx(row["porosity"], rel=1e-12)


def test_seeded_workloads_are_deterministic():
    a = designs.gyroid_design(0)
    b = designs.gyroid_design(0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    m, hs, u, info = a
    assert m.shape == (148, 128, 32) and 0.02 <= u <= 0.08 and 12 <= info["L"] <= 24
    assert (m[:, :, :4] == 1).all() and (m[0, 1:-1, 4:-1] == 2).all() and (m[-1, 1:-1, 4:-1] == 3).all()
    assert hs[:, :, 1:].max() == 0 and hs.max() > 0
    fams = {designs.mixed_design(s)[3]["family"] for s in range(10)}
    assert fams == set(designs.FAMILIES)


def test_straight_fin_plate_layout():
    m = designs.straight_fin_plate()
    assert m.shape == (64, 32, 16)
    assert (m[8:56, 4:6, 4:15] == 1).all() and (m[8:56, 6:9, 4:15] == 0).all()
    assert (m[0, 1:31, 4:15] == 2).all() and (m[63, 1:31, 4:15] == 3).all()


def _evaluate_spec(spec):
    """The per-cell rule of the device design kernel (csrc/designs.cu), restated in numpy for the parameters
    reference_spec produces: the same inputs must give the reference's masks without a GPU."""
    nx, ny, nz = spec["shape"]
    buf = spec["buf"]
    core = nx - 2 * buf
    p0, p1 = spec["p"]
    solid = np.zeros((core, ny, nz), dtype=bool)
    fam = spec["family"]
    if fam == "straight":
        designs._straight_channels(solid, int(p0), int(p1))
    elif fam == "pin_fin":
        X, Y = np.meshgrid(np.arange(core), np.arange(ny), indexing="ij")
        h, ip = p1 / 2, int(p1)
        da = ((X % ip) - h) ** 2 + ((Y % ip) - h) ** 2
        db = (np.mod(X - h, p1) - h) ** 2 + (np.mod(Y - h, p1) - h) ** 2
        solid[:] = (np.minimum(da, db) < p0 * p0)[:, :, None]
    elif fam in ("gyroid", "schwarz_p", "schwarz_d"):
        kind = {"gyroid": 3, "schwarz_p": 4, "schwarz_d": 5}[fam]
        f = designs.tpms_field(kind, (core, ny, nz), p0)
        solid[:] = (f < p1) if spec.get("below") else (f > p1)
        m = spec.get("margin", 0)
        if m:
            solid[:m] = False
            solid[-m:] = False
    mask = np.zeros((nx, ny, nz), dtype=np.int32)
    mask[buf:buf + core][solid] = designs.BC_SOLID
    return designs._frame(mask)


@pytest.mark.parametrize("case", D["masks"], ids=lambda c: "t{design_type}-{feature_size}-{spacing}".format(**c["state"]))
def test_reference_spec_reproduces_the_reference_masks(case):
    """reference_spec's parameters (what the device builder evaluates) give the reference's mask bytes."""
    m = _evaluate_spec(designs.reference_spec(case["state"]))
    assert sha(m.astype(np.int32)) == case["sha256"]
