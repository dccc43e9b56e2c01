"""Cold-plate design masks and heat maps (host-side input generation).

* ``generate_mask(state)`` restates src/geometry.py:339-526 (empty channel, straight channels, staggered
  pin fins, gyroid, Schwarz P and Schwarz D TPMS in a 128x128x32 core with 10-cell inlet/outlet buffers).
* ``HEAT_SOURCE_REGISTRY`` restates the ten floor heat maps of src/geometry.py:69-336.
* ``straight_fin_plate``, ``gyroid_design`` and ``mixed_design`` build the seeded synthetic workloads
  used by the tests and the benchmark: a 64x32x16 finned plate, a 148x128x32 gyroid with a seeded
  Gaussian-hotspot floor map, and uneven-size designs of five families.
"""
from __future__ import annotations

import numpy as np

BC_FLUID, BC_SOLID, BC_INLET, BC_OUTLET = 0, 1, 2, 3
CORE_NX, CORE_NY, CORE_NZ = 128, 128, 32  # src/geometry.py:15
DESIGN_NAMES = ["Empty Channel", "Straight Channels", "Pin-Fin Staggered", "Gyroid TPMS", "Schwarz P TPMS",
                "Schwarz D TPMS"]  # src/geometry.py:29
BASE_THICKNESS, TOP_THICKNESS = 4, 1  # src/geometry.py:516-517


def _frame(mask: np.ndarray) -> np.ndarray:
    """Side walls, base plate, lid, inlet and outlet planes (src/geometry.py:510-524)."""
    mask[:, 0, :] = BC_SOLID
    mask[:, -1, :] = BC_SOLID
    mask[:, :, :BASE_THICKNESS] = BC_SOLID
    mask[:, :, -TOP_THICKNESS:] = BC_SOLID
    mask[0, 1:-1, BASE_THICKNESS:-TOP_THICKNESS] = BC_INLET
    mask[-1, 1:-1, BASE_THICKNESS:-TOP_THICKNESS] = BC_OUTLET
    return mask


def _straight_channels(solid: np.ndarray, width: int, n_channels: int) -> None:
    """src/geometry.py:385-434: N channels of ``width`` separated by N+1 equal walls (the last wall fills)."""
    ny = solid.shape[1]
    total = n_channels * width
    if total >= ny:
        return
    gap = float(ny - total) / (n_channels + 1)
    y_end = int(gap)
    if y_end > 0:
        solid[:, :y_end, :] = True
    pos = gap
    for i in range(n_channels):
        pos += width
        y0 = int(pos)
        y1 = ny if i == n_channels - 1 else int(pos + gap)
        if y0 < ny:
            solid[:, y0:y1, :] = True
        pos += gap


def _pin_fins(solid: np.ndarray, raw_width: float, raw_count: float) -> None:
    """src/geometry.py:436-457: two interleaved square lattices of circular pins."""
    nx, ny, _ = solid.shape
    d_pin = max(2, int(raw_width * 2.0))
    pitch = max(d_pin + 2, int(raw_count * 3.0))
    radius = d_pin / 2.0
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    da = ((X % pitch) - pitch / 2) ** 2 + ((Y % pitch) - pitch / 2) ** 2
    db = (((X - pitch / 2) % pitch) - pitch / 2) ** 2 + (((Y - pitch / 2) % pitch) - pitch / 2) ** 2
    solid[:, :, :] = (np.minimum(da, db) < radius ** 2)[:, :, None]


def tpms_field(kind: int, shape, cell_size: float) -> np.ndarray:
    """Implicit TPMS value on the integer grid (src/geometry.py:476-495): 3 gyroid, 4 Schwarz P, 5 Schwarz D."""
    omega = 2.0 * np.pi / cell_size
    X, Y, Z = np.meshgrid(*(np.arange(s) for s in shape), indexing="ij")
    wx, wy, wz = X * omega, Y * omega, Z * omega
    if kind == 3:
        return np.sin(wx) * np.cos(wy) + np.sin(wy) * np.cos(wz) + np.sin(wz) * np.cos(wx)
    if kind == 4:
        return np.cos(wx) + np.cos(wy) + np.cos(wz)
    if kind == 5:
        return (np.sin(wx) * np.sin(wy) * np.sin(wz) + np.sin(wx) * np.cos(wy) * np.cos(wz)
                + np.cos(wx) * np.sin(wy) * np.cos(wz) + np.cos(wx) * np.cos(wy) * np.sin(wz))
    raise ValueError(f"unknown TPMS kind {kind}")


def _generate_params(state: dict):
    """src/geometry.py:339-379: (design, buffer, channel width, channel count, pin diameter, pin pitch, TPMS
    threshold C, TPMS cell size) from a GUI/sampler state."""
    design = min(max(int(state["design_type"]), 0), len(DESIGN_NAMES) - 1)
    buf = int(state["buffer_size"])
    raw_width = state.get("feature_size", 3.0)
    raw_count = state.get("spacing", 3.0)
    width = max(2, int(raw_width * 2.0))
    target = max(4, int(raw_count * 4.0))
    n_channels = max(2, min(target, int((CORE_NY - 1) / (width + 1))))
    d_pin = max(2, int(raw_width * 2.0))
    pitch = max(d_pin + 2, int(raw_count * 3.0))
    C = 0.8 - ((raw_width - 1.0) / 9.0) * 1.6
    cell_size = 20.0 + ((raw_count - 1.0) / 9.0) * 80.0
    return design, buf, width, n_channels, d_pin, pitch, C, cell_size


def reference_spec(state: dict) -> dict:
    """generate_mask's design as the parameters of the device evaluation (xadvcool_b200.device_designs):
    family, lattice shape, buffer, and the family's two numbers (channel width / count, pin radius / pitch, TPMS
    cell size / threshold with solid below it and 5 fluid x cells at each end of the core)."""
    design, buf, width, n_channels, d_pin, pitch, C, cell_size = _generate_params(state)
    spec = {"shape": (CORE_NX + 2 * buf, CORE_NY, CORE_NZ), "buf": buf, "hot": [], "background": 0.0}
    if design == 0:
        spec.update(family="empty", p=(0.0, 0.0))
    elif design == 1:
        spec.update(family="straight", p=(float(width), float(n_channels)))
    elif design == 2:
        spec.update(family="pin_fin", p=(d_pin / 2.0, float(pitch)))
    else:
        spec.update(family=["gyroid", "schwarz_p", "schwarz_d"][design - 3], p=(cell_size, C), below=True, margin=5)
    return spec


def generate_mask(state: dict) -> np.ndarray:
    """src/geometry.py:339-526 with ``state`` keys design_type, feature_size, spacing, buffer_size."""
    nx, ny, nz = CORE_NX, CORE_NY, CORE_NZ
    design, buf, width, n_channels, _, _, C, cell_size = _generate_params(state)
    mask = np.full((nx + 2 * buf, ny, nz), BC_FLUID, dtype=np.int32)
    solid = np.zeros((nx, ny, nz), dtype=bool)
    if design == 1:
        _straight_channels(solid, width, n_channels)
    elif design == 2:
        _pin_fins(solid, state.get("feature_size", 3.0), state.get("spacing", 3.0))
    elif design in (3, 4, 5):
        solid[:, :, :] = tpms_field(design, (nx, ny, nz), cell_size) < C
        solid[:5] = False
        solid[-5:] = False
    mask[buf:buf + nx][solid] = BC_SOLID
    return _frame(mask)


# ------------------------------------------------------------------------------------------------
# heat maps, src/geometry.py:69-336
def _blur_normalise(hm: np.ndarray, sigma: float) -> np.ndarray:
    from scipy import ndimage
    hm = ndimage.gaussian_filter(hm, sigma=sigma)
    if hm.max() > 0:
        hm /= hm.max()
    return hm


def _dual_core(nx, ny):
    hm = np.zeros((nx, ny), dtype=np.float32)
    hm[:, :] = 0.1
    hm[int(nx * 0.25):int(nx * 0.75), int(ny * 0.55):int(ny * 0.85)] = 1.0
    hm[int(nx * 0.25):int(nx * 0.75), int(ny * 0.15):int(ny * 0.45)] = 1.0
    hm[int(nx * 0.30):int(nx * 0.70), int(ny * 0.45):int(ny * 0.55)] = 0.5
    return _blur_normalise(hm, nx / 80.0)


def _quad_core(nx, ny):
    hm = np.full((nx, ny), 0.08, dtype=np.float32)
    for x0, y0, x1, y1 in ((0.15, 0.55, 0.45, 0.85), (0.15, 0.15, 0.45, 0.45), (0.55, 0.55, 0.85, 0.85),
                           (0.55, 0.15, 0.85, 0.45)):
        hm[int(nx * x0):int(nx * x1), int(ny * y0):int(ny * y1)] = 1.0
    hm[int(nx * 0.45):int(nx * 0.55), int(ny * 0.10):int(ny * 0.90)] = 0.45
    hm[int(nx * 0.10):int(nx * 0.90), int(ny * 0.45):int(ny * 0.55)] = 0.45
    return _blur_normalise(hm, nx / 80.0)


def _gpu_die(nx, ny):
    hm = np.full((nx, ny), 0.05, dtype=np.float32)
    hm[int(nx * 0.15):int(nx * 0.85), int(ny * 0.15):int(ny * 0.85)] = 0.75
    hm[int(nx * 0.10):int(nx * 0.90), int(ny * 0.02):int(ny * 0.12)] = 1.0
    hm[int(nx * 0.10):int(nx * 0.90), int(ny * 0.88):int(ny * 0.98)] = 1.0
    xx, yy = np.ogrid[:nx, :ny]
    for cxf in (0.30, 0.50, 0.70):
        cx, cy, r = int(nx * cxf), int(ny * 0.50), int(min(nx, ny) * 0.04)
        hm[(xx - cx) ** 2 + (yy - cy) ** 2 < r ** 2] = 1.0
    return _blur_normalise(hm, nx / 60.0)


def _chiplet(nx, ny):
    hm = np.full((nx, ny), 0.03, dtype=np.float32)
    w, h = 0.18, 0.22
    for x0, y0 in ((0.12, 0.08), (0.12, 0.40), (0.12, 0.72), (0.58, 0.08), (0.58, 0.40), (0.58, 0.72)):
        hm[int(nx * x0):int(nx * (x0 + w)), int(ny * y0):int(ny * (y0 + h))] = 1.0
    hm[int(nx * 0.38):int(nx * 0.52), int(ny * 0.10):int(ny * 0.90)] = 0.35
    return _blur_normalise(hm, nx / 70.0)


def _igbt(nx, ny):
    hm = np.full((nx, ny), 0.02, dtype=np.float32)
    for i, y0 in enumerate((0.05, 0.20, 0.38, 0.55, 0.72, 0.88)):
        if i % 2 == 0:
            hm[int(nx * 0.20):int(nx * (0.20 + 0.50)), int(ny * y0):int(ny * (y0 + 0.10))] = 1.0
        else:
            hm[int(nx * 0.30):int(nx * (0.30 + 0.25)), int(ny * y0):int(ny * (y0 + 0.10))] = 0.55
    return _blur_normalise(hm, nx / 60.0)


def _soc(nx, ny):
    hm = np.full((nx, ny), 0.06, dtype=np.float32)
    hm[int(nx * 0.10):int(nx * 0.35), int(ny * 0.60):int(ny * 0.90)] = 1.0
    for dy in (0.08, 0.22):
        for dx in (0.10, 0.28):
            hm[int(nx * dx):int(nx * (dx + 0.12)), int(ny * (0.35 + dy)):int(ny * (0.35 + dy + 0.10))] = 0.30
    hm[int(nx * 0.50):int(nx * 0.90), int(ny * 0.35):int(ny * 0.90)] = 0.65
    hm[int(nx * 0.05):int(nx * 0.95), int(ny * 0.02):int(ny * 0.12)] = 0.40
    hm[int(nx * 0.45):int(nx * 0.60), int(ny * 0.15):int(ny * 0.30)] = 0.80
    return _blur_normalise(hm, nx / 70.0)


def _gaussian_hotspots(nx, ny, seed=0):
    rng = np.random.RandomState(seed)
    hm = np.full((nx, ny), 0.05, dtype=np.float32)
    n = rng.randint(1, 4)
    xx, yy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    for _ in range(n):
        cx = rng.uniform(0.2, 0.8) * nx
        cy = rng.uniform(0.2, 0.8) * ny
        sigma = rng.uniform(0.06, 0.15) * min(nx, ny)
        amp = rng.uniform(0.5, 1.0)
        hm += amp * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * sigma ** 2))
    if hm.max() > 0:
        hm /= hm.max()
    return hm


def _hotspot_on_background(nx, ny):
    hm = np.full((nx, ny), 0.20, dtype=np.float32)
    xx, yy = np.ogrid[:nx, :ny]
    cx, cy, r = int(nx * 0.40), int(ny * 0.60), int(min(nx, ny) * 0.07)
    hm[(xx - cx) ** 2 + (yy - cy) ** 2 < r ** 2] = 1.0
    cx, cy, r = int(nx * 0.65), int(ny * 0.35), int(min(nx, ny) * 0.05)
    hm[(xx - cx) ** 2 + (yy - cy) ** 2 < r ** 2] = 0.85
    return _blur_normalise(hm, nx / 100.0)


def _peripheral_ring(nx, ny):
    hm = np.full((nx, ny), 0.05, dtype=np.float32)
    w = 0.10
    hm[:int(nx * w), :] = 0.85
    hm[int(nx * (1 - w)):, :] = 0.85
    hm[:, :int(ny * w)] = 0.85
    hm[:, int(ny * (1 - w)):] = 0.85
    r = int(min(nx, ny) * 0.12)
    xx, yy = np.ogrid[:nx, :ny]
    for cxf, cyf in ((0.0, 0.0), (0.0, 1.0), (1.0, 0.0), (1.0, 1.0)):
        cx, cy = int(nx * cxf), int(ny * cyf)
        hm[(xx - cx) ** 2 + (yy - cy) ** 2 < r ** 2] = 1.0
    hm[int(nx * 0.20):int(nx * 0.80), int(ny * 0.20):int(ny * 0.80)] = 0.15
    return _blur_normalise(hm, nx / 60.0)


HEAT_SOURCE_REGISTRY = {
    "uniform": lambda nx, ny, **kw: np.ones((nx, ny), dtype=np.float32),
    "dual_core": lambda nx, ny, **kw: _dual_core(nx, ny),
    "quad_core": lambda nx, ny, **kw: _quad_core(nx, ny),
    "gpu_die": lambda nx, ny, **kw: _gpu_die(nx, ny),
    "chiplet": lambda nx, ny, **kw: _chiplet(nx, ny),
    "igbt_half_bridge": lambda nx, ny, **kw: _igbt(nx, ny),
    "soc_heterogeneous": lambda nx, ny, **kw: _soc(nx, ny),
    "gaussian_hotspots": lambda nx, ny, **kw: _gaussian_hotspots(nx, ny, seed=kw.get("seed", 0)),
    "hotspot_on_background": lambda nx, ny, **kw: _hotspot_on_background(nx, ny),
    "peripheral_ring": lambda nx, ny, **kw: _peripheral_ring(nx, ny),
}
HEAT_SOURCE_NAMES = list(HEAT_SOURCE_REGISTRY.keys())


def floor_heat_source(shape, hs_2d: np.ndarray, buf: int = 10) -> np.ndarray:
    """3-D heat source with a 2-D map on the z=0 floor of the core (generate_dataset.py:404-410)."""
    nx, ny, nz = shape
    hs = np.zeros((nx, ny, nz), dtype=np.float32)
    cx, cy = hs_2d.shape
    hs[buf:buf + cx, :cy, 0] = hs_2d
    return hs


# ------------------------------------------------------------------------------------------------
# seeded synthetic workloads
def straight_fin_plate(nx=64, ny=32, nz=16, fins=((4, 6), (9, 11), (14, 16), (19, 21), (24, 26)),
                       x_range=(8, 56)) -> np.ndarray:
    """64x32x16 plate: side walls, 4-cell base plate, lid, inlet/outlet planes, and full-height fins
    2 cells wide with 3-cell gaps over x in [8, 56)."""
    mask = np.full((nx, ny, nz), BC_FLUID, dtype=np.int32)
    for y0, y1 in fins:
        mask[x_range[0]:x_range[1], y0:y1, :] = BC_SOLID
    return _frame(mask)


def draw_hotspots(rng: np.random.Generator, nx: int, ny: int):
    """K ~ U{1..4} Gaussian hotspots (cx, cy, sigma ~ U[4,12] cells, amplitude ~ U[0.5,1])."""
    out = []
    for _ in range(int(rng.integers(1, 5))):
        cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        sigma = rng.uniform(4.0, 12.0)
        amp = rng.uniform(0.5, 1.0)
        out.append((cx, cy, sigma, amp))
    return out


def hotspot_map(hot, nx: int, ny: int) -> np.ndarray:
    """0.2 background plus the given Gaussian hotspots, evaluated in float64, stored as float32."""
    hm = np.full((nx, ny), 0.2, dtype=np.float64)
    xx, yy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    for cx, cy, sigma, amp in hot:
        hm += amp * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2.0 * sigma ** 2))
    return hm.astype(np.float32)


def seeded_hotspot_map(rng: np.random.Generator, nx: int, ny: int) -> np.ndarray:
    """0.2 background plus K ~ U{1..4} Gaussian hotspots, sigma ~ U[4,12] cells, amplitude ~ U[0.5,1]."""
    return hotspot_map(draw_hotspots(rng, nx, ny), nx, ny)


def gyroid_spec(seed: int, nx=148, ny=128, nz=32, buf=10) -> dict:
    """The random draws of gyroid_design: L ~ U{12..24}, t ~ U[-0.4, 0.4], u_in ~ U[0.02, 0.08], then the
    hotspot map's draws. The returned spec also drives the device builder (xadvcool_b200.device_designs)."""
    rng = np.random.default_rng(seed)
    L = int(rng.integers(12, 25))
    t = float(rng.uniform(-0.4, 0.4))
    u_in = float(rng.uniform(0.02, 0.08))
    core = nx - 2 * buf
    return {"family": "gyroid", "shape": (nx, ny, nz), "buf": buf, "L": L, "t": t, "margin": 0, "u_in": u_in,
            "hot": draw_hotspots(rng, core, ny), "seed": seed}


def mixed_spec(seed: int, family: str | None = None) -> dict:
    """The random draws of mixed_design, in its order."""
    rng = np.random.default_rng(10_000 + seed)
    fam = family or FAMILIES[seed % len(FAMILIES)]
    nx = int(rng.choice([96, 128, 148, 192]))
    ny = int(rng.choice([64, 96, 128]))
    nz = int(rng.choice([16, 32, 48]))
    buf = 10
    core = nx - 2 * buf
    spec = {"family": fam, "shape": (nx, ny, nz), "buf": buf, "seed": seed, "margin": 0}
    if fam == "straight":
        n = int(rng.integers(4, 13))
        spec.update(n=n, width=max(2, (ny - 2) // (2 * n)))
    elif fam == "pin_fin":
        radius = int(rng.integers(2, 6))
        spec.update(radius=radius, pitch=int(rng.integers(max(8, 2 * radius + 2), 17)))
    else:
        spec.update(L=int(rng.integers(12, 25)), t=float(rng.uniform(-0.3, 0.3)), margin=5)
    spec["u_in"] = float(rng.uniform(0.02, 0.05))
    spec["hot"] = draw_hotspots(rng, core, ny)
    return spec


_TPMS_KIND = {"gyroid": 3, "schwarz_p": 4, "schwarz_d": 5}


def build_from_spec(spec: dict):
    """Host evaluation of a spec -> (mask int32 [nx][ny][nz], heat source float32 [nx][ny][nz])."""
    nx, ny, nz = spec["shape"]
    buf = spec["buf"]
    core = nx - 2 * buf
    fam = spec["family"]
    solid = np.zeros((core, ny, nz), dtype=bool)
    if fam == "straight":
        _straight_channels(solid, spec["width"], spec["n"])
    elif fam == "pin_fin":
        radius, pitch = spec["radius"], spec["pitch"]
        X, Y = np.meshgrid(np.arange(core), np.arange(ny), indexing="ij")
        da = ((X % pitch) - pitch / 2) ** 2 + ((Y % pitch) - pitch / 2) ** 2
        db = (((X - pitch / 2) % pitch) - pitch / 2) ** 2 + (((Y - pitch / 2) % pitch) - pitch / 2) ** 2
        solid[:, :, :] = (np.minimum(da, db) < radius ** 2)[:, :, None]
    else:
        solid = tpms_field(_TPMS_KIND[fam], (core, ny, nz), float(spec["L"])) > spec["t"]
        m = spec.get("margin", 0)
        if m:
            solid[:m] = False
            solid[-m:] = False
    mask = np.full((nx, ny, nz), BC_FLUID, dtype=np.int32)
    mask[buf:buf + core][solid] = BC_SOLID
    mask = _frame(mask)
    hs = floor_heat_source((nx, ny, nz), hotspot_map(spec["hot"], core, ny), buf=buf)
    return mask, hs


def gyroid_design(seed: int, nx=148, ny=128, nz=32, buf=10):
    """148x128x32 gyroid: solid where sin(kx)cos(ky)+sin(ky)cos(kz)+sin(kz)cos(kx) > t, k = 2pi/L,
    L ~ U{12..24}, t ~ U[-0.4, 0.4], in the core x in [buf, nx-buf), plus the reference frame
    (4-cell base plate, walls, inlet/outlet). Returns (mask, heat_source, u_inlet, info)."""
    spec = gyroid_spec(seed, nx, ny, nz, buf)
    mask, hs = build_from_spec(spec)
    return mask, hs, spec["u_in"], {"L": spec["L"], "t": spec["t"], "u_in": spec["u_in"], "seed": seed}


FAMILIES = ("straight", "pin_fin", "gyroid", "schwarz_p", "schwarz_d")


def mixed_design(seed: int, family: str | None = None):
    """One uneven-size design of the five families with x in {96,128,148,192}, y in {64,96,128},
    z in {16,32,48}: straight channels (n = 4..12), staggered pin fins (radius 2..5, pitch 8..16), gyroid,
    Schwarz P (cos+cos+cos > t) and Schwarz D. Returns (mask, heat_source, u_inlet, info)."""
    spec = mixed_spec(seed, family)
    mask, hs = build_from_spec(spec)
    info = {"family": spec["family"], "shape": spec["shape"], "seed": seed, "u_in": spec["u_in"]}
    for k in ("n", "width", "radius", "pitch", "L", "t"):
        if k in spec:
            info[k] = spec[k]
    return mask, hs, spec["u_in"], info
