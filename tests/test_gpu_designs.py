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
