"""Host-side helpers of bench.py: clock records, algorithmic bytes, ef choice,
the committed traffic figure. No GPU and no index needed."""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

IDLE = ["Not Active"] * 4


def test_clock_record_drops_the_sample_taken_before_the_timed_region():
    rows = [(1100.0, 1965.0, IDLE), (1965.0, 1965.0, IDLE), (1950.0, 1965.0, IDLE), (1965.0, 1965.0, IDLE)]
    rec = bench.summarize_clock_rows(rows)
    assert rec == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3}


def test_clock_record_keeps_a_lone_sample_and_reports_reasons():
    assert bench.summarize_clock_rows([]) is None
    assert bench.summarize_clock_rows([(1800.0, 1965.0, IDLE)])["samples"] == 1
    rows = [(1965.0, 1965.0, IDLE), (1300.0, 1965.0, ["Not Active", "Not Active", "Not Active", "Active"]),
            (1290.0, 1965.0, ["Active", "Not Active", "Not Active", "Active"])]
    rec = bench.summarize_clock_rows(rows)
    assert rec["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert rec["sm_mhz"] == 1295.0


def test_sampler_is_absent_without_nvidia_smi(tmp_path):
    # On a host without a GPU the sampler cannot start; timing goes on and
    # the record is null.
    r, clocks = bench.sampled(lambda: 7, tag="cpu-test")
    assert r == 7
    if not any(os.access(os.path.join(p, "nvidia-smi"), os.X_OK) for p in os.environ.get("PATH", "").split(":")):
        assert clocks is None


def test_algorithmic_bytes_per_query():
    # One query: 700 layer-0 distances, 60 layer-0 lists, 20 upper distances,
    # 5 upper lists, k = 10 (the per-unit figure the roofline uses).
    counters = np.array([[700, 60, 20, 5]], dtype=np.uint32)
    want = 4 * 128 * 720 + 4 * 33 * 60 + 4 * 17 * 5 + 4 * 128 + 12 * 10
    assert bench.algorithmic_bytes(counters, 10) == want
    assert bench.algorithmic_bytes(np.repeat(counters, 3, axis=0), 10) == 3 * want


def test_headline_ef_is_the_smallest_reaching_the_recall_target():
    assert bench.choose_ef({16: 0.70, 32: 0.87, 64: 0.966, 128: 0.99, 256: 0.998}) == 64
    assert bench.choose_ef({16: 0.1, 32: 0.2, 64: 0.3, 128: 0.4, 256: 0.5}) == 256


def test_committed_traffic_figure_is_read():
    t = bench.profiled_traffic()
    assert t is not None and 1e9 < t < 1e11
