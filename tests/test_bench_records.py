"""The records bench.py reads on the GPU box (no GPU needed): the recorded DRAM
traffic of each line's dominant kernel, keyed by workload, and the measured peaks
it divides by."""

import json
from pathlib import Path

import bench

ROOT = Path(__file__).resolve().parent.parent


def test_recorded_traffic_keys():
    rec = json.loads((ROOT / "profiles" / "traffic.json").read_text())
    for key in ("combined_512_1920x1080", "per_source_bf16_512_1920x1080", "learned_half_512_960x540", "batch_512_4"):
        assert isinstance(rec[key], int) and rec[key] > 0, key
        assert bench.recorded_traffic(key) == rec[key]
    # the headline launch reads its 2.53 GB brick texture about once
    assert 2.0e9 < rec["combined_512_1920x1080"] < 3.5e9
    assert bench.recorded_traffic("no such workload") is None


def test_measured_peaks_are_read():
    peak, kind = bench.measured_peaks()
    assert peak > 1000.0 and kind in ("measured", "fallback")
    allp = bench.measured_peaks_all()
    assert allp["hbm_gbs"] == peak and allp["bf16_tflops"] > 100.0
