"""The seeded benchmark designs built on the GPU (xac_design_build): the same random draws as
xadvcool_b200.designs (gyroid_spec / mixed_spec, numpy's generator on the host) with the per-cell evaluation -
TPMS field, channel walls, pin lattices, frame and Gaussian-hotspot floor map - done by a CUDA kernel.

    mask, heat, u_in, info = gyroid_design(0)        # torch tensors on the GPU, reference layout [nx][ny][nz]
    mask, heat = reference_design({"design_type": 3, "feature_size": 5.0, "spacing": 3.0, "buffer_size": 10},
                                  "chiplet")        # the reference's generate_mask families
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from . import designs as _host
from ._tensors import stream_ptr


def spec_struct(spec: dict) -> _capi.DesignSpec:
    nx, ny, nz = spec["shape"]
    fam = spec["family"]
    if "p" in spec:
        p0, p1 = spec["p"]
    elif fam == "straight":
        p0, p1 = spec["width"], spec["n"]
    elif fam == "pin_fin":
        p0, p1 = spec["radius"], spec["pitch"]
    else:
        p0, p1 = spec["L"], spec["t"]
    code = _capi.DESIGN_FAMILIES[fam] | (_capi.DESIGN_BELOW if spec.get("below") else 0)
    s = _capi.DesignSpec(nx, ny, nz, spec["buf"], code, spec.get("margin", 0), float(p0), float(p1),
                         len(spec["hot"]), float(spec.get("background", 0.2)))
    for k, h in enumerate(spec["hot"]):
        for j in range(4):
            s.hot[k][j] = float(h[j])
    return s


def build(spec: dict, device="cuda"):
    """-> (mask int32, heat source float32) CUDA tensors [nx][ny][nz]."""
    dev = torch.device(device)
    nx, ny, nz = spec["shape"]
    mask = torch.empty((nx, ny, nz), dtype=torch.int32, device=dev)
    heat = torch.empty((nx, ny, nz), dtype=torch.float32, device=dev)
    s = spec_struct(spec)
    with torch.cuda.device(dev):
        _capi.call("xac_design_build", ctypes.byref(s), mask.data_ptr(), heat.data_ptr(), stream_ptr(dev))
    return mask, heat


def reference_design(state: dict, heat_source_type: str | None = None, seed: int = 0, device="cuda"):
    """generate_mask(state) (src/geometry.py:339-526) evaluated on the GPU, and optionally one of the ten floor
    heat maps (src/geometry.py:69-336; 128x128, built on the host, where it takes about a millisecond) placed on
    the core floor as generate_dataset.py:404-410 does. -> (mask int32, heat source float32) CUDA tensors."""
    spec = _host.reference_spec(state)
    mask, heat = build(spec, device)
    if heat_source_type is not None:
        hm = _host.HEAT_SOURCE_REGISTRY[heat_source_type](_host.CORE_NX, _host.CORE_NY, seed=seed)
        b = spec["buf"]
        heat[b:b + hm.shape[0], :hm.shape[1], 0] = torch.from_numpy(np.ascontiguousarray(hm, np.float32)).to(heat.device)
    return mask, heat


def gyroid_design(seed: int, nx=148, ny=128, nz=32, buf=10, device="cuda"):
    spec = _host.gyroid_spec(seed, nx, ny, nz, buf)
    mask, heat = build(spec, device)
    return mask, heat, spec["u_in"], {"L": spec["L"], "t": spec["t"], "u_in": spec["u_in"], "seed": seed}


def mixed_design(seed: int, family: str | None = None, device="cuda"):
    spec = _host.mixed_spec(seed, family)
    mask, heat = build(spec, device)
    info = {"family": spec["family"], "shape": spec["shape"], "seed": seed, "u_in": spec["u_in"]}
    return mask, heat, spec["u_in"], info
