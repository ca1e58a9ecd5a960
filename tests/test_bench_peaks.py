"""bench.py reads the HBM roofline denominator from MEASURED_PEAKS.json in
whatever numeric shape it is written, and falls back (labelled) instead of
failing when the file is missing, unreadable or holds no HBM figure."""
import json

import pytest


@pytest.mark.parametrize("content, expected", [
    ({"hbm_gbs": 7012.5, "bf16_tflops": 1590.0}, 7012.5),
    ({"hbm_gbs": "7012.5"}, 7012.5),
    ({"hbm_gbs": {"value": 7012.5, "unit": "GB/s"}}, 7012.5),
    ({"hbm_gbs": {"burst": 7100, "sustained": 6900}}, 7100.0),
    ({"hbm_GBps": 6900}, 6900.0),
])
def test_measured_peak_shapes(tmp_path, content, expected):
    import bench
    p = tmp_path / "MEASURED_PEAKS.json"
    p.write_text(json.dumps(content))
    assert bench.load_peaks(str(p)) == (expected, "measured")


@pytest.mark.parametrize("text", ["not json", json.dumps({"bf16_tflops": 1590.0}), json.dumps({"hbm_gbs": None}),
                                  json.dumps({"hbm_gbs": -1}), json.dumps([7000])])
def test_unusable_peaks_fall_back(tmp_path, text):
    import bench
    p = tmp_path / "MEASURED_PEAKS.json"
    p.write_text(text)
    value, kind = bench.load_peaks(str(p))
    assert value == bench.FALLBACK_HBM_GBS and kind.startswith("fallback")


def test_missing_peaks_fall_back(tmp_path):
    import bench
    assert bench.load_peaks(str(tmp_path / "absent.json")) == (bench.FALLBACK_HBM_GBS, "fallback")
