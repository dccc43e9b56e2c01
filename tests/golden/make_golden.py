"""Generate tests/golden/*.json from the reference checkout (run in a container that has it; the GPU box
does not, so the outputs are committed).

* designs.json  — sha256 of generate_mask() for the parameters of selected dataset rows and of a grid of
                  states, and of the ten heat maps (src/geometry.py, imported with a pyvista stub).
* metrics.json  — compute_macroscopic_metrics() (generate_dataset.py:80-179, imported with h5py and
                  src.simulation stubs) on seeded synthetic fields (fields rebuilt by ``synthetic_fields``).
* validate.json — validate_sample() (analyze_dataset.py:184-323, imported with h5py and matplotlib stubs; the
                  HDF5 group is served from memory) on the seeded cases of oracle.validate_ref.validation_case.
* parquet_rows.json — stratified rows of dataset/metadata.parquet (inputs and golden scalars of the
                  reference's GPU runs), excluding gaussian_hotspots rows whose seed is process-salted.
* failed_rows.json — stratified entries of dataset/failed_samples.json (designs the reference rejected as
                  invalid geometry, diverged or unphysical) with their parameters, recovered by regenerating the
                  reference's sample list (generate_samples, 200 per design, seed 42: the dataset's 10,000 ids,
                  every failed id among them) and hashing each parameter set into its sample id as
                  generate_dataset.py:368-369 does. Solved designs exclude gaussian_hotspots heat maps.

Usage: python tests/golden/make_golden.py REFERENCE_DIR   (or XAC_REFERENCE_DIR=REFERENCE_DIR)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))  # the repository root: oracle/ and xadvcool_b200/


def synthetic_fields(seed: int, shape=(148, 128, 32)):
    """Smooth seeded fields in the ranges of converged solutions (rho ~ 1, |u| < 0.1, T in 25..40)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x = np.linspace(0, 1, nx)[:, None, None]
    y = np.linspace(0, 1, ny)[None, :, None]
    z = np.linspace(0, 1, nz)[None, None, :]
    a = rng.uniform(0.5, 2.0, size=8)
    rho = (1.0 + 0.01 * a[0] * (1 - x) + 0.002 * np.sin(6 * a[1] * y) * np.cos(5 * z)).astype(np.float32)
    u = np.zeros((nx, ny, nz, 3), dtype=np.float32)
    u[..., 0] = 0.03 * a[2] * np.sin(np.pi * y) * np.sin(np.pi * z) + 0.001 * np.cos(7 * a[3] * x)
    u[..., 1] = 0.005 * np.sin(9 * a[4] * x) * np.cos(4 * y)
    u[..., 2] = 0.004 * np.cos(5 * a[5] * x) * np.sin(3 * z)
    T = (25.0 + 10.0 * a[6] * (1 - z) * np.exp(-3 * (y - 0.5) ** 2) + 2.0 * a[7] * x).astype(np.float32)
    T = np.broadcast_to(T, (nx, ny, nz)).copy()
    rho = np.broadcast_to(rho, (nx, ny, nz)).copy()
    return rho, u, T


def validation_case(seed: int):
    """A seeded small gyroid design with smooth fields consistent with solver output (solid rho = 1, u = 0),
    its heat map normalised to 1, and fixed dataset attributes."""
    from xadvcool_b200.designs import gyroid_design
    mask, hs, u_in, _ = gyroid_design(seed, nx=48, ny=24, nz=16, buf=6)
    rho, u, T = synthetic_fields(100 + seed, shape=mask.shape)
    solid = mask == 1
    rho[solid] = 1.0
    u[solid] = 0.0
    hs = (hs / hs.max()).astype(np.float32)
    attrs = {"heat_power": 0.1, "Pr": 7.0, "k_ratio": 628.0, "tau_fluid": 0.55, "Nu": 12.5 + seed,
             "f_friction": 0.8, "Re": 30.0 + seed}
    return mask, rho, u, T, hs, attrs


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _import_reference(ref: Path):
    sys.path.insert(0, str(ref))
    sys.modules.setdefault("pyvista", types.ModuleType("pyvista"))
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    sim = types.ModuleType("src.simulation")
    sim.run_simulation = None
    sys.modules["src.simulation"] = sim
    import src.geometry as geometry  # noqa: E402
    import generate_dataset as gd  # noqa: E402
    return geometry, gd


def _validate_reference(ref: Path):
    """analyze_dataset.validate_sample with its HDF5 reader and plotting imports stubbed: the returned function
    runs the reference code on in-memory arrays."""
    sys.path.insert(0, str(ref))
    store = {}

    class _Ds:
        def __init__(self, a):
            self.a = a

        def __getitem__(self, k):
            return self.a

    class _Grp:
        def __init__(self, d, attrs):
            self.d, self.attrs = d, attrs

        def __getitem__(self, k):
            return _Ds(self.d[k])

    class _File:
        def __init__(self, path, mode="r"):
            self.path = path

        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

        def __getitem__(self, sid):
            d, attrs = store[sid]
            return _Grp(d, attrs)

    h5 = types.ModuleType("h5py")
    h5.File = _File
    sys.modules["h5py"] = h5
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    mpl.rcParams = {}
    sys.modules["matplotlib"] = mpl
    for sub in ("pyplot", "ticker", "colors", "gridspec", "cm", "patches", "lines", "collections"):
        m = types.ModuleType("matplotlib." + sub)
        m.__getattr__ = lambda name: object  # any plotting name imports as a placeholder
        setattr(mpl, sub, m)
        sys.modules["matplotlib." + sub] = m
    import analyze_dataset as ad  # noqa: E402

    def run(mask, rho, u, T, hs, attrs):
        store["s"] = ({"mask": mask, "velocity": u, "temperature": T, "pressure": rho / 3.0, "heat_source": hs},
                      dict(attrs))
        return ad.validate_sample("unused.h5", "s")

    return run


def sample_id(params: dict) -> str:
    """generate_dataset.py:366-369."""
    ps = json.dumps(params, sort_keys=True) + "|coolant=water"
    return f"{params['design_name'].replace(' ', '_')}_water_{hashlib.md5(ps.encode()).hexdigest()[:8]}"


def write_failed_rows(ref: Path, gd):
    failed = json.loads((ref / "dataset" / "failed_samples.json").read_text())
    found = {}
    for name in gd.DESIGN_CONFIGS:
        for params in gd.generate_samples(name, 200, seed=42):
            found[sample_id(params)] = params
    missing = [k for k in failed if k not in found]
    assert not missing, f"{len(missing)} failed ids not in the regenerated sample list"
    by = {}
    for sid, reason in sorted(failed.items()):
        p = found[sid]
        cat = reason.split(" (")[0]
        if cat != "invalid geometry" and p["heat_source_type"] == "gaussian_hotspots":
            continue  # heat map seeded by the process-salted hash(sample_id)
        by.setdefault((p["design_name"], cat), []).append((sid, reason, p))
    quota = {"invalid geometry": 6, "diverged": 2, "unphysical": 2}
    rng = np.random.default_rng(4321)
    out = []
    for (name, cat), lst in sorted(by.items()):
        for i in sorted(rng.choice(len(lst), size=min(quota[cat], len(lst)), replace=False).tolist()):
            sid, reason, p = lst[i]
            out.append({"sample_id": sid, "category": cat, "reason": reason, "params": p})
    (HERE / "failed_rows.json").write_text(json.dumps(out, indent=1, sort_keys=True))
    return len(out)


def main(ref: Path):
    import pandas as pd
    geometry, gd = _import_reference(ref)
    df = pd.read_parquet(ref / "dataset" / "metadata.parquet")

    # ---- parquet rows: stratified over design family x heat map, reproducible heat maps only
    rows = []
    rng = np.random.default_rng(1234)
    keep = df[df["heat_source_type"] != "gaussian_hotspots"]
    for (design, hs), grp in keep.groupby(["design_name", "heat_source_type"]):
        pick = grp.iloc[int(rng.integers(0, len(grp)))]
        rows.append(pick)
    cols = ["sample_id", "design_name", "design_idx", "heat_source_type", "feature_size", "spacing", "tau_fluid",
            "u_inlet_val", "heat_power", "Pr", "k_ratio", "porosity", "Dh", "Re", "max_velocity", "max_temperature",
            "mean_temperature", "pressure_drop", "sim_steps", "converged", "R_th", "Nu", "f_friction", "P_pump",
            "COP", "Q_vol", "T_max_surface", "T_avg_surface", "delta_T_max", "sigma_T", "fluid_temp_rise",
            "elapsed_s", "mlups"]
    out_rows = []
    for r in rows:
        d = {c: (r[c].item() if hasattr(r[c], "item") else r[c]) for c in cols}
        state = {"design_type": d["design_idx"], "feature_size": d["feature_size"], "spacing": d["spacing"],
                 "buffer_size": 10}
        mask = geometry.generate_mask(state)
        d["mask_sha256"] = _sha(mask.astype(np.int32))
        d["porosity_check"] = float(gd.compute_porosity(mask))
        Dh, V, A = gd.compute_hydraulic_diameter(mask)
        d["Dh_check"], d["V_fluid"], d["A_wetted"] = float(Dh), int(V), int(A)
        out_rows.append(d)
    (HERE / "parquet_rows.json").write_text(json.dumps(out_rows, indent=1, sort_keys=True))

    # ---- designs: a grid of states per family plus every selected row
    states = []
    for t in range(6):
        for fs in (1.5, 3.3, 5.0, 8.5):
            for sp in (1.5, 2.7, 6.0):
                states.append({"design_type": t, "feature_size": fs, "spacing": sp, "buffer_size": 10})
    designs = []
    for s in states:
        m = geometry.generate_mask(s)
        designs.append({"state": s, "shape": list(m.shape), "sha256": _sha(m.astype(np.int32)),
                        "n_solid": int((m == 1).sum())})
    heat = {}
    for name, fn in geometry.HEAT_SOURCE_REGISTRY.items():
        seeds = (0, 1, 7) if name == "gaussian_hotspots" else (0,)
        for sd in seeds:
            hm = fn(128, 128, seed=sd).astype(np.float32)
            heat[f"{name}:{sd}"] = {"sha256": _sha(hm), "sum": float(hm.astype(np.float64).sum()),
                                    "max": float(hm.max()), "probe": [float(hm[17, 33]), float(hm[64, 64]),
                                                                      float(hm[101, 90])]}
    (HERE / "designs.json").write_text(json.dumps({"masks": designs, "heat_maps": heat}, indent=1))

    # ---- metrics: the reference function on seeded fields over three masks
    mcases = []
    for k, s in enumerate([{"design_type": 1, "feature_size": 3.3, "spacing": 2.7, "buffer_size": 10},
                           {"design_type": 2, "feature_size": 2.5, "spacing": 4.0, "buffer_size": 10},
                           {"design_type": 3, "feature_size": 6.0, "spacing": 3.0, "buffer_size": 10}]):
        mask = geometry.generate_mask(s)
        rho, u, T = synthetic_fields(100 + k, mask.shape)
        params = {"tau_fluid": 0.53 + 0.01 * k, "u_inlet_val": 0.02 + 0.01 * k}
        Dh, V, A = gd.compute_hydraulic_diameter(mask)
        res = gd.compute_macroscopic_metrics({"u": u, "rho": rho, "T": T}, mask, params, Dh, A, Pr=7.0)
        mcases.append({"state": s, "seed": 100 + k, "params": params, "Dh": float(Dh), "A_wetted": int(A),
                       "V_fluid": int(V), "porosity": float(gd.compute_porosity(mask)),
                       "pressure_drop_all": float(np.mean(rho[1]) - np.mean(rho[-2])) / 3.0,
                       "metrics": {k2: float(v) for k2, v in res.items()}})
    (HERE / "metrics.json").write_text(json.dumps(mcases, indent=1))

    # ---- validators: the reference's validate_sample on seeded small designs (oracle.validate_ref.validation_case)
    run = _validate_reference(ref)
    vcases = []
    for seed in range(3):
        mask, rho, u, T, hs, attrs = validation_case(seed)
        res = run(mask, rho, u, T, hs, attrs)
        vcases.append({"seed": seed, "checks": {k: (bool(v) if isinstance(v, (bool, np.bool_)) else float(v))
                                                for k, v in res.items() if k != "sample_id"}})
    (HERE / "validate.json").write_text(json.dumps(vcases, indent=1))
    n_failed = write_failed_rows(ref, gd)
    print(f"wrote {len(out_rows)} rows, {len(designs)} masks, {len(heat)} heat maps, {len(mcases)} metric cases, "
          f"{n_failed} failed-sample rows")


if __name__ == "__main__":
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("XAC_REFERENCE_DIR")
    if not ref_dir:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_DIR  (or set XAC_REFERENCE_DIR): the path of "
                 "the reference checkout whose geometry, metrics and validator code generate the fixtures")
    main(Path(ref_dir))
