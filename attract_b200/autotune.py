"""Launch-shape autotuner for the persistent minimiser.

Candidates are (lanes per pose, threads per block): 8/16/32 lanes per pose
(4/2/1 poses per warp) x 64/128 threads.  Each candidate minimises a sample
of every segment for a few steps, timed with CUDA events; the fastest wins and
is cached in a JSON file (``$ATTRACT_B200_CACHE`` or
``~/.cache/attract_b200/autotune.json``) under a key of what decides the
winner: the GPU, the ligand bead counts, and a binned histogram of the
grids' neighbour-list lengths (long lists shift the balance between the
per-bead and the per-pair work).
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from ._lib import AttractError
from .engine import AdamOptions, EvalOptions, LaunchShape, Segment, Workload, minimise

CANDIDATES = [(8, 64), (8, 128), (16, 64), (16, 128), (32, 64), (32, 128)]
# list-length bins of the cache key: empty, 1-5, 6-10, 11-20, 21-40, more
LIST_BINS = (0, 1, 6, 11, 21, 41)


def _cache_path() -> str:
    return os.environ.get("ATTRACT_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "attract_b200",
                                                              "autotune.json"))


def list_histogram(counts) -> tuple:
    """Fractions of list-grid points per LIST_BINS bin, rounded to 0.05 so that
    receptors of the same kind share a key."""
    c = np.asarray(counts, np.int64).reshape(-1)
    if c.size == 0:
        return tuple(0.0 for _ in LIST_BINS)
    idx = np.searchsorted(np.asarray(LIST_BINS), c, side="right") - 1
    frac = np.bincount(idx, minlength=len(LIST_BINS)) / c.size
    return tuple(float(round(f * 20) / 20) for f in frac)


def grid_list_histogram(grid) -> tuple:
    """:func:`list_histogram` of a Grid's neighbour lists (cached on the grid)."""
    h = getattr(grid, "_list_hist", None)
    if h is None:
        if grid.nb_hdr is None:
            h = list_histogram([])
        else:
            cnt = grid.nb_hdr[:, 1].to(torch.int64)
            edges = torch.tensor(LIST_BINS[1:], dtype=torch.int64, device=cnt.device)
            idx = torch.bucketize(cnt, edges, right=True)
            frac = torch.bincount(idx, minlength=len(LIST_BINS)).cpu().numpy() / max(cnt.numel(), 1)
            h = tuple(float(round(f * 20) / 20) for f in frac)
        grid._list_hist = h
    return h


def cache_key(device_name: str, bead_sizes, list_hists) -> str:
    """The autotuner's cache key: GPU, sorted distinct bead counts, and the
    list-length histogram of every grid the workload uses."""
    sizes = ",".join(str(int(n)) for n in sorted(set(int(x) for x in bead_sizes)))
    hists = ";".join(",".join(f"{f:.2f}" for f in h) for h in list_hists)
    return f"{device_name}|beads={sizes}|lists={hists}"


def _key(wl: Workload) -> str:
    name = torch.cuda.get_device_name(wl.device)
    sizes = [wl.ligands.sizes[s.lig] for s in wl.segments if s.n_poses]
    used = sorted(set(s.grid for s in wl.segments if s.n_poses))
    return cache_key(name, sizes, [grid_list_histogram(wl.grids[g]) for g in used])


def cache_lookup(path: str, key: str):
    """(LaunchShape, timings) cached under ``key`` in ``path``, or None."""
    if not os.path.exists(path):
        return None
    try:
        hit = json.load(open(path)).get(key)
    except (OSError, ValueError):
        return None
    if not hit:
        return None
    return LaunchShape(int(hit["lanes"]), int(hit["threads"])), hit.get("ms", {})


def cache_store(path: str, key: str, shape: LaunchShape, times: dict) -> None:
    """Add or replace ``key`` in the JSON cache file (other keys are kept)."""
    try:
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        try:
            data = json.load(open(path)) if os.path.exists(path) else {}
        except ValueError:
            data = {}
        data[key] = dict(lanes=shape.lanes_per_pose, threads=shape.block_threads, ms=times)
        tmp = path + ".tmp"
        json.dump(data, open(tmp, "w"), indent=1)
        os.replace(tmp, path)
    except OSError:
        pass


def autotune(wl: Workload, poses: torch.Tensor, steps: int = 10, sample: int = 65536,
             adam: AdamOptions | None = None, opts: EvalOptions | None = None, use_cache: bool = True,
             candidates=CANDIDATES, repeats: int = 2) -> tuple[LaunchShape, dict]:
    """Pick the fastest launch shape for ``wl``; returns (shape, timings in ms)."""
    key = _key(wl)
    path = _cache_path()
    if use_cache:
        hit = cache_lookup(path, key)
        if hit is not None:
            return hit
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
    shape = LaunchShape(lanes, threads)
    if use_cache:
        cache_store(path, key, shape, times)
    return shape, times
