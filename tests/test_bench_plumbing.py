"""bench.py's roofline inputs read on the host: the HBM peak (MEASURED_PEAKS.json, else the stated fallback) and
the DRAM traffic per cell-step from the committed ncu summary of the step kernel."""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_traffic_comes_from_the_committed_profile_of_the_same_kernel_and_shape():
    text = (ROOT / "profiles" / "coupled_step_gyroid148.md").read_text()
    assert f"profiled_sources_sha256: {bench.step_sources_sha256()}" in text
    for block in (64, 128, 256):
        tpc, why = bench.ncu_traffic_per_cell(block, 0)
        assert why is None and 150.0 < tpc < 320.0  # between the solid-aware and the all-cell algorithmic bytes
    tpc, why = bench.ncu_traffic_per_cell(96, 0)
    assert tpc is None and "no figure" in why


def test_traffic_is_withheld_for_other_kernel_sources(tmp_path, monkeypatch):
    prof = tmp_path / "profiles"
    prof.mkdir()
    text = (ROOT / "profiles" / "coupled_step_gyroid148.md").read_text()
    (prof / "coupled_step_gyroid148.md").write_text(text.replace(bench.step_sources_sha256(), "0" * 64))
    src = tmp_path / "xadvcool_b200" / "csrc"
    src.mkdir(parents=True)
    for name in bench.STEP_SOURCES:
        (src / name).write_bytes((ROOT / "xadvcool_b200" / "csrc" / name).read_bytes())
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    tpc, why = bench.ncu_traffic_per_cell(128, 0)
    assert tpc is None and "other step kernel sources" in why


def test_peak_is_measured_or_the_stated_fallback(tmp_path, monkeypatch):
    peak, kind = bench.hbm_peak()
    assert kind in ("measured", "fallback") and peak > 1000.0
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.hbm_peak() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6549.8}))
    assert bench.hbm_peak() == (6549.8, "measured")
