"""The launch-shape autotuner's cache key and cache file (no GPU needed)."""
import json

import numpy as np


def test_list_histogram_bins_and_rounding():
    from attract_b200.autotune import LIST_BINS, list_histogram

    counts = np.array([0] * 50 + [3] * 20 + [8] * 10 + [15] * 10 + [30] * 5 + [70] * 5)
    h = list_histogram(counts)
    assert len(h) == len(LIST_BINS)
    assert h == (0.5, 0.2, 0.1, 0.1, 0.05, 0.05)
    assert abs(sum(h) - 1.0) < 1e-9
    assert list_histogram([]) == tuple(0.0 for _ in LIST_BINS)
    # bins are [0], [1, 5], [6, 10], [11, 20], [21, 40], [41, ...)
    assert list_histogram([5]) == (0.0, 1.0, 0.0, 0.0, 0.0, 0.0)
    assert list_histogram([6]) == (0.0, 0.0, 1.0, 0.0, 0.0, 0.0)
    assert list_histogram([41]) == (0.0, 0.0, 0.0, 0.0, 0.0, 1.0)


def test_cache_key_names_gpu_beads_and_list_histogram():
    from attract_b200.autotune import cache_key

    h1 = (0.5, 0.4, 0.1, 0.0, 0.0, 0.0)
    h2 = (0.2, 0.3, 0.2, 0.2, 0.05, 0.05)
    k = cache_key("NVIDIA B200", [30, 18, 24, 18], [h1])
    assert k == cache_key("NVIDIA B200", [18, 24, 30], [h1])  # order and repeats do not matter
    assert k != cache_key("NVIDIA B200", [18, 24, 30], [h2])  # long lists: another key
    assert k != cache_key("NVIDIA H100", [18, 24, 30], [h1])
    assert k != cache_key("NVIDIA B200", [18, 24], [h1])
    assert "beads=18,24,30" in k and "lists=0.50,0.40,0.10" in k


def test_cache_file_round_trip(tmp_path):
    from attract_b200.autotune import cache_lookup, cache_store
    from attract_b200.engine import LaunchShape

    path = str(tmp_path / "sub" / "autotune.json")
    assert cache_lookup(path, "k1") is None
    cache_store(path, "k1", LaunchShape(32, 128), {"32x128": 1.5, "8x64": 2.0})
    cache_store(path, "k2", LaunchShape(8, 64), {"8x64": 0.7})
    shape, times = cache_lookup(path, "k1")
    assert (shape.lanes_per_pose, shape.block_threads) == (32, 128) and times["8x64"] == 2.0
    shape, _ = cache_lookup(path, "k2")
    assert (shape.lanes_per_pose, shape.block_threads) == (8, 64)
    cache_store(path, "k1", LaunchShape(16, 64), {})  # replaced, k2 kept
    data = json.load(open(path))
    assert data["k1"]["lanes"] == 16 and data["k2"]["lanes"] == 8
    open(path, "w").write("{not json")  # a corrupt file is a miss, and is rewritten
    assert cache_lookup(path, "k1") is None
    cache_store(path, "k3", LaunchShape(32, 64), {})
    assert cache_lookup(path, "k3")[0].lanes_per_pose == 32
