"""Launch-shape autotuner for the persistent minimiser.

Candidates are (lanes per pose, threads per block): 8/16/32 lanes per pose
(4/2/1 poses per warp) x 64/128 threads.  Each candidate minimises a sample
of every segment for a few steps, timed with CUDA events; the fastest wins and
is cached per (GPU, bead-count histogram) in a JSON file
(``$ATTRACT_B200_CACHE`` or ``~/.cache/attract_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from ._lib import AttractError
from .engine import AdamOptions, EvalOptions, LaunchShape, Segment, Workload, minimise

CANDIDATES = [(8, 64), (8, 128), (16, 64), (16, 128), (32, 64), (32, 128)]


def _cache_path() -> str:
    return os.environ.get("ATTRACT_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "attract_b200",
                                                              "autotune.json"))


def _key(wl: Workload) -> str:
    name = torch.cuda.get_device_name(wl.device)
    sizes = sorted(set(int(wl.ligands.sizes[s.lig]) for s in wl.segments if s.n_poses))
    return f"{name}|{','.join(map(str, sizes))}"


def autotune(wl: Workload, poses: torch.Tensor, steps: int = 10, sample: int = 65536,
             adam: AdamOptions | None = None, opts: EvalOptions | None = None, use_cache: bool = True,
             candidates=CANDIDATES, repeats: int = 2) -> tuple[LaunchShape, dict]:
    """Pick the fastest launch shape for ``wl``; returns (shape, timings in ms)."""
    key = _key(wl)
    path = _cache_path()
    if use_cache and os.path.exists(path):
        try:
            hit = json.load(open(path)).get(key)
            if hit:
                return LaunchShape(hit["lanes"], hit["threads"]), hit.get("ms", {})
        except (OSError, ValueError):
            pass
    # a sample of each segment, same bead-count mix
    segs, parts = [], []
    for s, p0 in zip(wl.segments, wl.pose0):
        k = min(s.n_poses, max(1, sample * s.n_poses // max(wl.n_poses, 1)))
        segs.append(Segment(s.grid, s.lig, k))
        parts.append(poses[p0:p0 + k])
    sp = torch.cat(parts).contiguous()
    times = {}
    for lanes, threads in candidates:
        w = Workload(wl.grids, wl.ligands, segs, lanes, wl.device)
        shape = LaunchShape(lanes, threads)
        try:
            minimise(w, sp, 1, adam, opts, launch=shape)  # warm
        except AttractError as e:
            if "shared memory" not in str(e):
                raise
            continue  # this block size cannot hold the beads per lane this ligand mix needs
        best = float("inf")
        for _ in range(repeats):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            minimise(w, sp, steps, adam, opts, launch=shape)
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        times[f"{lanes}x{threads}"] = best
    if not times:
        raise AttractError("no candidate launch shape fits this workload's shared memory")
    lanes, threads = (int(x) for x in min(times, key=times.get).split("x"))
    if use_cache:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            data = json.load(open(path)) if os.path.exists(path) else {}
            data[key] = dict(lanes=lanes, threads=threads, ms=times)
            json.dump(data, open(path, "w"), indent=1)
        except (OSError, ValueError):
            pass
    return LaunchShape(lanes, threads), times
