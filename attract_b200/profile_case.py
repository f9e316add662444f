"""Run the batched minimiser on a synthetic workload a few times (for profilers).

    python -m attract_b200.profile_case [--config 1] [--scale 0.05] [--types 32]
        [--launches 3] [--lanes 32] [--threads 64] [--steps N] [--refine 4]

Builds the workload (grid build, neighbour lists, bricks), then launches the
persistent minimisation kernel ``--launches`` times and prints the mean time of
the launches after the first.  ``--types`` shrinks the number of ligand types
(and so the grid) to keep profiler captures small.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--scale", type=float, default=0.05)
    ap.add_argument("--types", type=int, default=32)
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--lanes", type=int, default=32)
    ap.add_argument("--threads", type=int, default=64)
    ap.add_argument("--steps", type=int, default=-1)
    ap.add_argument("--refine", type=int, default=4, help="neighbour-list grid refinement (1, 2 or 4)")
    a = ap.parse_args()

    import attract_b200 as A
    from attract_b200 import synth

    A.load_library()
    cfg = synth.make_config(a.config, seed=0, scale=a.scale, n_types=a.types)
    steps = cfg.steps if a.steps < 0 else a.steps
    grid = A.Grid.build(cfg.rec_xyz, cfg.rec_type, cfg.ff, cfg.geom, cutoff=cfg.cutoff, nb_refine=a.refine)
    ligs = A.LigandSet(cfg.ligands)
    order = sorted(range(len(cfg.ligands)), key=lambda i: -len(cfg.ligands[i][0]))
    wl = A.Workload([grid], ligs, [A.Segment(0, i, len(cfg.poses[i])) for i in order], lanes_per_pose=a.lanes)
    poses = torch.tensor(np.concatenate([cfg.poses[i] for i in order]).astype(np.float32), device="cuda")
    shape = A.LaunchShape(a.lanes, a.threads)
    scratch = A.MinimiseScratch(wl.n_poses, wl.device)
    out = torch.empty_like(poses)
    times = []
    for i in range(a.launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        A.minimise(wl, poses, steps, pose_out=out, launch=shape, scratch=scratch)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    _, _, _, st = A.minimise(wl, poses, steps, launch=shape, stats=True)
    st = st.cpu().numpy().tolist()
    ms = float(np.mean(times[1:])) if len(times) > 1 else times[0]
    print(json.dumps({"config": a.config, "scale": a.scale, "types": a.types, "poses": wl.n_poses, "steps": steps,
                      "lanes": a.lanes, "threads": a.threads, "ms": ms, "poses_per_s": wl.n_poses / ms * 1e3,
                      "stats": st, "brick_gb": grid.bricks.numel() * 4 / 1e9}))


if __name__ == "__main__":
    main()
