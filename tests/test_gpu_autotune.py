"""The launch-shape autotuner on the GPU: the shape it picks runs the
workload, and is reused from the cache on the next call with the same key."""
import numpy as np
import pytest
import torch

from gpu_cases import small_case, to_device_grid

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_fitting_shape_and_reuses_the_cache(tmp_path, monkeypatch):
    import attract_b200 as A
    from attract_b200 import autotune as T

    A.load_library()
    monkeypatch.setenv("ATTRACT_B200_CACHE", str(tmp_path / "autotune.json"))
    c = small_case(seed=70, n_poses=600)
    grid = to_device_grid(c)
    rng = np.random.default_rng(1)
    lig2 = rng.normal(size=(21, 3)) * 2.0  # a second fragment of another size
    t2 = rng.integers(0, c["n_types"], 21)
    ligs = A.LigandSet([(c["lig"], c["gt"], c["lt"]), (lig2, t2, t2)])
    wl = A.Workload([grid], ligs, [A.Segment(0, 0, 300), A.Segment(0, 1, 300)])
    P = torch.tensor(c["poses"][np.r_[0:300, 0:300]], dtype=torch.float32, device="cuda")
    shape, times = T.autotune(wl, P, steps=3, sample=256)
    assert f"{shape.lanes_per_pose}x{shape.block_threads}" in times
    assert len(times) >= 3  # several candidates fitted and were timed
    key = T._key(wl)
    assert "lists=" in key and "beads=9,21" in key
    hit = T.cache_lookup(str(tmp_path / "autotune.json"), key)
    assert hit is not None and hit[0].lanes_per_pose == shape.lanes_per_pose
    # the second call is served from the cache (no candidate is run)
    calls = []
    monkeypatch.setattr(T, "minimise", lambda *a, **k: calls.append(1))
    shape2, _ = T.autotune(wl, P, steps=3, sample=256)
    assert calls == [] and (shape2.lanes_per_pose, shape2.block_threads) == (shape.lanes_per_pose,
                                                                                shape.block_threads)
    # the picked shape runs the workload; the block size does not change a
    # pose's arithmetic, so the other block size gives the same result bit for bit
    wt = wl.with_lanes(shape.lanes_per_pose)
    out, E, S, _ = A.minimise(wt, P, 5, launch=shape)
    other = A.LaunchShape(shape.lanes_per_pose, 64 if shape.block_threads == 128 else 128)
    out2, E2, _, _ = A.minimise(wt, P, 5, launch=other)
    assert torch.equal(E, E2) and torch.equal(out, out2)
    assert torch.all(S == 0)
