"""Continuous-batching server: a request's result is the same alone and in a
mix of receptors, ligand sizes and arrival times; rounds equal one launch."""
import numpy as np
import pytest
import torch

from gpu_cases import small_case, to_device_grid

pytestmark = pytest.mark.gpu


def _server(grids, **kw):
    import attract_b200 as A
    from attract_b200.serve import DockingServer

    A.load_library()
    return DockingServer(grids, **kw)


def _req(seed, receptor, n_beads, n_poses):
    from attract_b200.serve import Request

    rng = np.random.default_rng(seed)
    lig = rng.normal(size=(n_beads, 3)) * 1.5
    lig -= lig.mean(0)
    t = rng.integers(0, 4, n_beads)
    poses = small_case(seed=100 + seed, n_poses=n_poses)["poses"].astype(np.float32)
    return Request(receptor, (lig, t, t), poses)


@pytest.fixture(scope="module")
def grids():
    return [to_device_grid(small_case(seed=s, n_poses=4)) for s in (40, 41, 42)]


def test_result_alone_equals_result_in_the_mix(grids):
    alone = _server(grids, steps=40, round_steps=10, max_inflight_poses=5000)
    a = alone.submit(_req(1, 1, 13, 70))
    alone.run_until_idle()
    mix = _server(grids, steps=40, round_steps=10, max_inflight_poses=5000)
    others = [mix.submit(_req(2, 0, 5, 40)), mix.submit(_req(3, 2, 30, 90))]
    mix.round()                       # the others are on the GPU ...
    b = mix.submit(_req(1, 1, 13, 70))  # ... when the request arrives
    mix.submit(_req(4, 1, 22, 33))
    mix.round()
    mix.submit(_req(5, 0, 9, 51))
    mix.run_until_idle()
    assert b.result_poses is not None and all(o.result_poses is not None for o in others)
    assert np.array_equal(a.result_poses, b.result_poses)
    assert np.array_equal(a.result_energies, b.result_energies)
    st = mix.stats()
    assert st["requests"] == 5 and st["p99_s"] >= st["p50_s"] > 0


@pytest.mark.parametrize("concurrent", [True, False])
def test_alone_equals_mix_across_launch_shapes(grids, concurrent):
    """Requests of different launch shapes (lanes per pose picked per ligand
    size, 1 and 2 beads per lane) in the same rounds: each result equals the
    request's result alone, bit for bit, whether the shape groups run on
    their own streams or one after another."""
    lanes_for = lambda n: 8 if n <= 8 else (16 if n <= 16 else 32)
    specs = [(30, 0, 6, 50), (31, 1, 60, 45), (32, 2, 14, 70), (33, 1, 27, 40), (34, 0, 40, 33)]
    alone = {}
    for sp in specs:
        srv = _server(grids, steps=30, round_steps=10, max_inflight_poses=5000, lanes_for=lanes_for)
        r = srv.submit(_req(*sp))
        srv.run_until_idle()
        alone[sp] = r
    mix = _server(grids, steps=30, round_steps=10, max_inflight_poses=5000, lanes_for=lanes_for,
                  concurrent=concurrent)
    got = {sp: mix.submit(_req(*sp)) for sp in specs[:3]}
    mix.round()
    got.update({sp: mix.submit(_req(*sp)) for sp in specs[3:]})
    mix.run_until_idle()
    assert {mix.shape_of(sp[2]) for sp in specs} == {(8, 1), (32, 2), (16, 1), (32, 1)}
    assert mix.stats()["launches"] > mix.stats()["rounds"]
    for sp in specs:
        assert np.array_equal(alone[sp].result_poses, got[sp].result_poses), sp
        assert np.array_equal(alone[sp].result_energies, got[sp].result_energies), sp


def test_rounds_equal_one_launch(grids):
    import attract_b200 as A

    srv = _server(grids, steps=40, round_steps=10, max_inflight_poses=5000)
    r = srv.submit(_req(6, 2, 17, 64))
    srv.run_until_idle()
    lig = r.ligand
    wl = A.Workload([grids[2]], A.LigandSet([lig]), [A.Segment(0, 0, 64)], lanes_per_pose=32)
    out, E, _, _ = A.minimise(wl, torch.tensor(r.poses, device="cuda"), 40, launch=A.LaunchShape(32))
    assert np.allclose(out.cpu().numpy(), r.result_poses, rtol=1e-5, atol=1e-5)
    assert np.allclose(E.cpu().numpy(), r.result_energies, rtol=1e-4, atol=1e-4)


def test_pool_admission_and_recycling(grids):
    srv = _server(grids, steps=20, round_steps=10, max_inflight_poses=100)
    reqs = [srv.submit(_req(10 + i, i % 3, 8, 60)) for i in range(4)]  # 240 poses, pool of 100
    srv.round()
    assert len(srv.active) == 1 and len(srv.pending) == 3
    srv.run_until_idle()
    assert all(r.result_energies is not None and np.all(np.isfinite(r.result_energies)) for r in reqs)
    assert srv.pool.used == 0
    with pytest.raises(ValueError):
        srv.submit(_req(20, 0, 8, 101))


def test_snapshot_resume_and_request_log(grids, tmp_path):
    """Stop a server between rounds, rebuild it from its snapshot and finish:
    every request's result equals an uninterrupted run's, bit for bit; each
    finished request leaves one JSON line in the log."""
    import json

    from attract_b200.serve import DockingServer

    reqs = [(7, 0, 11, 50), (8, 1, 24, 70), (9, 2, 6, 40)]
    full = _server(grids, steps=40, round_steps=10, max_inflight_poses=5000)
    ref = [full.submit(_req(*q)) for q in reqs]
    full.run_until_idle()

    log = tmp_path / "requests.jsonl"
    a = _server(grids, steps=40, round_steps=10, max_inflight_poses=5000, log_path=str(log))
    for q in reqs[:2]:
        a.submit(_req(*q))
    a.round()
    a.round()                      # two requests half way (20 of 40 steps) ...
    a.submit(_req(*reqs[2]))       # ... one still pending
    snap = a.snapshot()
    assert len(snap["requests"]) == 3 and snap["requests"][0]["step"] == 20
    b = DockingServer.resume(grids, snap, max_inflight_poses=3000, log_path=str(log))
    b.run_until_idle()
    got = sorted(b.done, key=lambda r: r.step0 == 0)  # the resumed pair first, then the pending one
    for r_ref, r in zip(ref, got):
        assert np.array_equal(r_ref.result_poses, r.result_poses)
        assert np.array_equal(r_ref.result_energies, r.result_energies)
    lines = [json.loads(x) for x in log.read_text().splitlines()]
    assert len(lines) == 3
    assert all(x["poses"] in (50, 70, 40) and x["latency_s"] >= 0 and x["flagged_poses"] == 0 for x in lines)
