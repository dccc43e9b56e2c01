"""bench.py's roofline inputs read on the host: the HBM peak (MEASURED_PEAKS.json, else the stated fallback) and
the DRAM traffic per cell-step from the committed ncu summary of the step kernel."""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_traffic_comes_from_the_committed_profile():
    text = (ROOT / "profiles" / "coupled_step_gyroid148.md").read_text()
    assert "dram_bytes_per_cell_step:" in text
    tpc = bench.ncu_traffic_per_cell()
    assert tpc is not None and 150.0 < tpc < 320.0  # between the solid-aware and the all-cell algorithmic bytes


def test_peak_is_measured_or_the_stated_fallback(tmp_path, monkeypatch):
    peak, kind = bench.hbm_peak()
    assert kind in ("measured", "fallback") and peak > 1000.0
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.hbm_peak() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6549.8}))
    assert bench.hbm_peak() == (6549.8, "measured")
