"""Designs built on the GPU (xac_design_build) against the host builder (xadvcool_b200.designs) for the same
seeds: identical masks, and heat maps equal up to the last float32 bit the device's exp may round differently."""
import numpy as np
import pytest

from xadvcool_b200 import designs as H
from xadvcool_b200 import device_designs as G

pytestmark = pytest.mark.gpu


def _same(dev, host):
    mask, heat = (t.cpu().numpy() for t in dev[:2])
    assert np.array_equal(mask, host[0])
    h = np.asarray(host[1], np.float32)
    # exp/sin/cos in double may differ from the host's by an ulp; after the float32 rounding that is at most
    # one float32 ulp, and almost always none
    assert np.all(np.abs(heat - h) <= np.spacing(np.abs(h)))
    assert dev[2] == host[2]


@pytest.mark.parametrize("seed", range(4))
def test_gyroid_matches_host(seed, cuda):
    _same(G.gyroid_design(seed), H.gyroid_design(seed))


@pytest.mark.parametrize("seed", range(15))
def test_mixed_families_match_host(seed, cuda):
    _same(G.mixed_design(seed), H.mixed_design(seed))


def test_rejects_bad_spec(cuda):
    spec = H.gyroid_spec(0)
    spec["hot"] = spec["hot"] * 3  # more hotspots than the spec holds
    spec["hot"] = spec["hot"][:9] if len(spec["hot"]) >= 9 else spec["hot"] + [(1.0, 1.0, 4.0, 0.5)] * 9
    with pytest.raises(Exception):
        G.build(spec)


# ---- the reference's generate_mask families (src/geometry.py:339-526) on the device
import hashlib  # noqa: E402
import json  # noqa: E402
from pathlib import Path  # noqa: E402

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "designs.json").read_text())
ROWS = json.loads((Path(__file__).resolve().parent / "golden" / "parquet_rows.json").read_text())


def _sha(t):
    return hashlib.sha256(np.ascontiguousarray(t.cpu().numpy().astype(np.int32)).tobytes()).hexdigest()


def test_reference_families_match_the_reference_masks(cuda):
    """All 72 golden states (6 design types x 4 feature sizes x 3 spacings), hashed from the reference's own
    generate_mask: the device mask has the same bytes."""
    bad = [m["state"] for m in GOLD["masks"] if _sha(G.reference_design(m["state"])[0]) != m["sha256"]]
    assert not bad, bad


def test_dataset_rows_build_on_the_device(cuda):
    """The 45 dataset rows' masks (hashed from the reference) and their floor heat maps."""
    for r in ROWS:
        state = {"design_type": r["design_idx"], "feature_size": r["feature_size"], "spacing": r["spacing"],
                 "buffer_size": 10}
        mask, heat = G.reference_design(state, r["heat_source_type"])
        assert _sha(mask) == r["mask_sha256"], r["sample_id"]
        host = H.floor_heat_source(tuple(mask.shape), H.HEAT_SOURCE_REGISTRY[r["heat_source_type"]](128, 128))
        assert np.array_equal(heat.cpu().numpy(), host)


def test_reference_design_rejects_bad_family(cuda):
    spec = H.reference_spec({"design_type": 1, "feature_size": 3.0, "spacing": 3.0, "buffer_size": 10})
    spec["below"] = True  # only TPMS families take the below-threshold convention
    with pytest.raises(Exception):
        G.build(spec)
