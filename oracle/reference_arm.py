"""CPU reference arm of bench.py (``--impl reference``).

TEST/BENCH INFRASTRUCTURE.  The reference (sjdv1982/attract-jax) is JAX and
cannot run here (no jax/optax anywhere in the image), so the reference arm
times the oracle's NumPy restatement of its minimiser (test5.py / test4.py
path, ``attract_oracle.minimise`` in float32) on every host core.  Nothing here
touches the GPU or the attract_b200 kernels: the grid is built by the oracle's
own CPU builder, in parallel, before timing.

Each timed step minimises a bounded sample of the benchmark workload (the same
receptor, fragments and poses; ``n`` poses of every fragment per worker) for
the full number of ADAM steps; the result is poses/s over the sample.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time
from multiprocessing import shared_memory

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

import attract_oracle as O  # noqa: E402


def _cfg(scale):
    from attract_b200 import synth  # NumPy input generation only

    return synth.make_config(1, seed=0, scale=scale)


def _build_chunk(args):
    shm_name, shape, lo, hi, rec, rtype, pair, geom, n_types, cutoff, outer = args
    shm = shared_memory.SharedMemory(name=shm_name)
    arr = np.ndarray(shape, np.float32, buffer=shm.buf)
    arr[:, lo:hi] = O.build_potential_grid(rec, rtype, pair, geom, n_types, cutoff, outer, (lo, hi))
    del arr
    shm.close()
    return hi - lo


def _minimise_task(args):
    names, shapes, geom, rec, rtype, pair, hdr, lst, ligs, poses, steps, lr_rot, lr_trans = args
    shms = [shared_memory.SharedMemory(name=n) for n in names]
    inner = np.ndarray(shapes[0], np.float32, buffer=shms[0].buf)
    outer = np.ndarray(shapes[1], np.float32, buffer=shms[1].buf)
    G = dict(geom=geom, inner=inner, outer=outer, nb_hdr=hdr, nb_list=lst, rec=rec, rtype=rtype, pair=pair)
    n = 0
    for (xyz, gt, lt), p in zip(ligs, poses):
        O.minimise(p, xyz, gt, lt, G, steps, lr_rot, lr_trans, dtype=np.float32)
        n += len(p)
    del inner, outer, G
    for s in shms:
        s.close()
    return n


def run(steps, warmup, metric, unit, workload, scale=1.0, per_worker=4):
    cfg = _cfg(scale)
    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    geom = cfg.geom.as_dict()
    pair = O.pair_table(cfg.ff.rc, cfg.ff.ac, cfg.ff.ivor, cfg.geom.plateau, True, cfg.ff.rcap2)
    rec = np.asarray(cfg.rec_xyz, np.float32).astype(np.float64)
    T = cfg.geom.n_types
    ctx = mp.get_context("spawn")
    shms, shapes = [], []
    t_build = time.perf_counter()
    with ctx.Pool(ncpu) as pool:
        for outer in (False, True):
            dims = tuple(int(x) for x in (geom["dim2"] if outer else geom["dim"]))
            npts = int(np.prod(dims))
            shape = (T, npts, 4)
            shm = shared_memory.SharedMemory(create=True, size=int(np.prod(shape)) * 4)
            step = (npts + 4 * ncpu - 1) // (4 * ncpu)
            tasks = [(shm.name, shape, lo, min(lo + step, npts), rec, cfg.rec_type, pair, geom, T, cfg.cutoff, outer)
                     for lo in range(0, npts, step)]
            pool.map(_build_chunk, tasks)
            shms.append(shm)
            shapes.append((T,) + dims + (4,))
        hdr, lst = O.build_nbgrid(rec, geom, cfg.geom.plateau + cfg.geom.spacing * np.sqrt(3) / 2 + 1e-3)
        build_s = time.perf_counter() - t_build
        ligs = [(np.asarray(x, np.float32).astype(np.float64), gt, lt) for x, gt, lt in cfg.ligands]
        tasks = []
        for w in range(ncpu):
            poses = [p[w * per_worker:(w + 1) * per_worker].astype(np.float32).astype(np.float64) for p in cfg.poses]
            tasks.append(([s.name for s in shms], shapes, geom, rec, cfg.rec_type, pair, hdr, lst, ligs, poses,
                          cfg.steps, cfg.lr_rot, cfg.lr_trans))
        times = []
        n = 0
        for i in range(warmup + steps):
            t = time.perf_counter()
            n = sum(pool.map(_minimise_task, tasks))
            dt = time.perf_counter() - t
            if i >= warmup:
                times.append(dt)
    for s in shms:
        s.close()
        s.unlink()
    ms = 1e3 * float(np.mean(times))
    value = n / (ms / 1e3)
    sample = (f"{n} poses ({per_worker} of each of the 6 fragments per worker, {ncpu} spawn workers) x "
              f"{cfg.steps} ADAM steps + final eval, NumPy float32 restatement of the reference path "
              "(jax/optax absent); grid built on the CPU by the oracle builder in "
              f"{build_s:.0f} s before timing")
    return {"metric": metric, "value": round(value, 2), "unit": unit, "n_gpus": 0, "steps": steps, "warmup": warmup,
            "ms_per_step": round(ms, 1), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded; no public dataset)", "impl": "reference",
            "config": {"workload": workload, "scale": scale, "sample_poses_per_step": n},
            "cpu_baseline": {"value": round(value, 2), "unit": unit, "cores": ncpu, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 2), "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
