"""Host-side pieces of bench.py (CPU only): the DRAM-traffic figure read from
the committed minimiser profile, the algorithmic-byte count of the roofline,
and the headline summary that the bench line ends with."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_profile_traffic_line_parses_and_scales(bench):
    per = bench.traffic_from_profile(1)
    assert per is not None, "profiles/minimise_kernel_config1.txt lost its dram_bytes_per_bead_eval line"
    # DRAM bytes per bead evaluation: far below the 128 algorithmic bytes of a brick read
    assert 1.0 < per < 128.0
    assert bench.traffic_from_profile(1000) == pytest.approx(1000 * per)


def test_algorithmic_bytes_per_bead_lookup_and_entry(bench):
    # 128 B per brick read, 8 B per list lookup, 2 B per list entry
    assert bench.algorithmic_bytes([1, 0, 0]) == 128
    assert bench.algorithmic_bytes([0, 1, 0]) == 8
    assert bench.algorithmic_bytes([0, 0, 1]) == 2
    assert bench.algorithmic_bytes([10, 10, 52]) == 1280 + 80 + 104


def test_summary_carries_the_headline_figures(bench):
    out = {"value": 4.6e6, "e2e": {"value": 4.58e6}, "roofline": {"frac": 0.505},
           "plain": {"value": 1.16e6}, "batched_vs_plain": 3.96,
           "cpu_baseline": {"value": 145.29},
           "configs": {"config2": {"value": 8.9e6, "bead_fraction_with_lists": 0.829, "list_length_max": 12},
                       "schema": {"fused": {"value": 2.1e6}}},
           "serving": {"runs": [{"arrival_rate_per_s": 200.0, "poses_per_s": 2.83e6, "p50_s": 10.1,
                                 "p99_s": 18.3, "backlog_requests": 3743}]}}
    sm = bench.summary(out)
    assert sm["batched_poses_per_s"] == 4.6e6 and sm["roofline_frac"] == 0.505
    assert sm["batched_vs_plain"] == 3.96
    assert sm["config2_value"] == 8.9e6 and sm["config2_bead_fraction_with_lists"] == 0.829
    assert sm["schema_value"] == 2.1e6
    assert sm["serving0"]["rate"] == 200.0 and sm["serving0"]["backlog_requests"] == 3743
