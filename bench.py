#!/usr/bin/env python
"""Benchmark of the batched rigid-body minimiser (one JSON line on stdout).

Workload (one "step"): the batched uneven-fragment minimisation -- a 2500-bead
synthetic receptor, 6 fragments of 18/21/24/26/28/30 beads, 100 000 poses
each (600 000 poses), 200 ADAM steps + a final evaluation, all fragments in
one persistent, CUDA-graph-captured launch.  ``value`` = minimised poses/s with
the inputs resident in HBM; ``e2e`` = the same through the public API with the
poses copied from pinned host memory and the energies + poses copied back
inside the timed region.  The 5.7 GB brick grid is larger than L2, so no L2
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): every rank minimises its own copy of the workload (replicas,
weak scaling); the time is the max over ranks.  ``--impl reference`` times the
CPU restatement of the reference path (oracle/, NumPy) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "minimised poses/s/GPU (200 ADAM steps), batched+served vs plain; p99 latency"
UNIT = "poses/s"
WORKLOAD = ("config1 batched uneven: receptor 2500 beads (40 A sphere, 32 types), fragments of "
            "18/21/24/26/28/30 beads x 100000 poses, 200 ADAM steps + final eval, fp32")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="pose-count scale (1 = the full workload)")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--cpu-poses", type=int, default=128, help="poses per fragment in the CPU sample")
    ap.add_argument("--no-configs", action="store_true", help="skip the other workloads (configs 0, 2, 3)")
    ap.add_argument("--serve-seconds", type=float, default=120.0,
                    help="length of the serving run (0 = skip; the full serving workload is 600 s)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="request arrivals per second")
    ap.add_argument("--serve-round-steps", type=int, default=50,
                    help="ADAM steps per serving round (a divisor of the 200 steps of a request)")
    ap.add_argument("--profile-case", action="store_true",
                    help="run only the minimiser on one configuration, --launches times (for ncu captures)")
    ap.add_argument("--config", type=int, default=1, help="--profile-case: configuration (0, 1 or 2)")
    ap.add_argument("--clustered", action="store_true", help="--profile-case: config 2's clustered receptor")
    ap.add_argument("--types", type=int, default=32, help="--profile-case: ligand types (grid size)")
    ap.add_argument("--launches", type=int, default=3, help="--profile-case: minimiser launches")
    ap.add_argument("--refine", type=int, default=4, help="--profile-case: neighbour-list grid refinement")
    ap.add_argument("--adam-steps", type=int, default=-1, help="--profile-case: ADAM steps (-1: the config's)")
    ap.add_argument("--allpairs", action="store_true",
                    help="--profile-case: the all-pairs rescoring kernel on config 3's receptor and ligand instead")
    return ap.parse_args()


# --------------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling (200 ms) while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = np.array([float(r[1]) for r in rows])
        mx = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        load = sm[sm > 0.5 * sm.max()] if len(sm) else sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows),
                "power_w_max": float(max(float(r[3]) for r in rows))}


# --------------------------------------------------------------------------- workload
def build(args, device):
    import torch

    import attract_b200 as A
    from attract_b200 import synth

    cfg = synth.make_config(1, seed=0, scale=args.scale)
    grid = A.Grid.build(cfg.rec_xyz, cfg.rec_type, cfg.ff, cfg.geom, cutoff=cfg.cutoff, keep_dense=not args.no_cpu,
                        device=device)
    ligs = A.LigandSet(cfg.ligands, device=device)
    order = sorted(range(len(cfg.ligands)), key=lambda i: -len(cfg.ligands[i][0]))  # largest first
    segs = [A.Segment(0, i, len(cfg.poses[i])) for i in order]
    poses = np.concatenate([cfg.poses[i] for i in order]).astype(np.float32)
    return cfg, grid, ligs, segs, poses, order


def algorithmic_bytes(stats):
    """128 B per grid-brick read + 8 B per list header + 2 B per list entry."""
    return int(stats[0]) * 128 + int(stats[1]) * 8 + int(stats[2]) * 2


def plain_run(A, grid, cfg, order, poses_np, steps, device):
    """The reference's call pattern on the GPU: one ligand at a time, one
    energy+gradient launch per step, ADAM in torch ops on the host side."""
    import torch

    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    off = 0
    launches = 0
    t0.record()
    for i in order:
        n = len(cfg.poses[i])
        wl = A.Workload([grid], A.LigandSet([cfg.ligands[i]], device=device), [A.Segment(0, 0, n)])
        x = torch.tensor(poses_np[off:off + n], device=device)
        off += n
        m = torch.zeros_like(x)
        v = torch.zeros_like(x)
        lr = torch.tensor([cfg.lr_rot] * 3 + [cfg.lr_trans] * 3, device=device)
        for s in range(1, steps + 1):
            E, g, _ = A.energrad(wl, x)
            launches += 1
            m.mul_(0.9).add_(g, alpha=0.1)
            v.mul_(0.999).addcmul_(g, g, value=0.001)
            mh = m / (1 - 0.9 ** s)
            vh = v / (1 - 0.999 ** s)
            x = x - lr * mh / (vh.sqrt() + 1e-8)
        E, _, _ = A.energrad(wl, x, grad=False)
        launches += 1
    t1.record()
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / 1e3, launches


def cpu_baseline(cfg, grid, order, n_per_frag, steps):
    """The oracle (NumPy float32, one process) on a bounded sample: the first
    n_per_frag poses of every fragment, the full step count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import attract_oracle as O

    inner, outer, hdr, lst = grid.dense_host()
    G = dict(geom=dict(cfg.geom.as_dict(), nb_refine=grid.nb_refine), inner=inner, outer=outer, nb_hdr=hdr, nb_list=lst,
             rec=np.asarray(cfg.rec_xyz, np.float32), rtype=cfg.rec_type,
             pair=O.pair_table(cfg.ff.rc, cfg.ff.ac, cfg.ff.ivor, cfg.geom.plateau, True, cfg.ff.rcap2))
    t = time.perf_counter()
    n = 0
    for i in order:
        xyz, gt, lt = cfg.ligands[i]
        p = cfg.poses[i][:n_per_frag]
        O.minimise(p, np.asarray(xyz, np.float32), gt, lt, G, steps, cfg.lr_rot, cfg.lr_trans, dtype=np.float32)
        n += len(p)
    dt = time.perf_counter() - t
    return {"value": n / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} poses ({n_per_frag} per fragment) x {steps} ADAM steps, NumPy float32 oracle, "
                      f"1 process, {dt:.1f} s"}


def traffic_from_profile(n_launch_units):
    """DRAM bytes per launch from the committed ncu summary, scaled to this
    launch by bead evaluations (the capture ran a smaller case)."""
    path = os.path.join(ROOT, "profiles", "minimise_kernel_config1.txt")
    if not os.path.exists(path):
        return None
    vals = {}
    for line in open(path):
        if "=" in line and line.strip().startswith("dram_bytes_per_bead_eval"):
            vals["per"] = float(line.split("=")[1].split()[0])
    if "per" not in vals:
        return None
    return vals["per"] * n_launch_units


# --------------------------------------------------------------------------- other workloads
def _timed(fn, reps, warm=2):
    import torch

    for _ in range(warm):
        fn()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def _peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    return float(json.load(open(p)).get("hbm_gbs", 6650.0)) if os.path.exists(p) else 6650.0


def other_configs(args, device, shape):
    """Plain small (config 0), neighbour-list heavy (config 2) and the
    differentiation workload (config 3), each on its own synthetic receptor."""
    import torch

    import attract_b200 as A
    from attract_b200 import synth
    from attract_b200.autograd import docking_energy
    from attract_b200.autotune import autotune
    from attract_b200.poses import euler_to_Q

    res = {}
    names = {"config0": "plain small: 1200-bead receptor, 7-bead fragment, 4096 poses, 1 eval + 100 ADAM steps",
             "config2": "nbgrid-heavy: 5000 beads at 0.01/A^3 (uniform, 3.5 A apart), 40-bead ligand, 500000 poses "
                        "with the centroid within 2 A of the solvent-accessible surface (probe 1.4 A + bead 2.0 A, "
                        "outer envelope and cavities), 1 eval + 50 ADAM",
             "config2_clustered": "nbgrid-heavy, clustered: the same 5000 beads in 40 dense patches (Gaussian, "
                                  "3 A wide, 1.5 A apart) at the same mean density, so lists of 0-80 entries; "
                                  "40-bead ligand, 500000 surface poses, 1 eval + 50 ADAM"}
    for key, idx, clustered in (("config0", 0, False), ("config2", 2, False), ("config2_clustered", 2, True)):
        cfg = synth.make_config(idx, seed=0, scale=args.scale, clustered=clustered)
        grid = A.Grid.build(cfg.rec_xyz, cfg.rec_type, cfg.ff, cfg.geom, cutoff=cfg.cutoff, device=device)
        ligs = A.LigandSet(cfg.ligands, device=device)
        poses_np = np.concatenate(cfg.poses).astype(np.float32)
        poses = torch.tensor(poses_np, device=device)
        wl = A.Workload([grid], ligs, [A.Segment(0, i, len(p)) for i, p in enumerate(cfg.poses)])
        shp, _ = autotune(wl, poses, use_cache=False)
        wl = wl.with_lanes(shp.lanes_per_pose)
        _, _, _, st = A.minimise(wl, poses, cfg.steps, launch=shp, stats=True)
        stats = st.cpu().numpy()
        scratch = A.MinimiseScratch(wl.n_poses, device)
        out = torch.empty_like(poses)
        ms = _timed(lambda: A.minimise(wl, poses, cfg.steps, launch=shp, pose_out=out, scratch=scratch), 5)
        e = {"workload": names[key], "poses": wl.n_poses, "adam_steps": cfg.steps,
             "value": round(wl.n_poses / ms * 1e3, 1), "unit": UNIT, "ms": round(ms, 3),
             "launch": {"lanes_per_pose": shp.lanes_per_pose},
             "roofline_frac": round(algorithmic_bytes(stats) / (ms / 1e3) / 1e9 / _peak(), 4),
             "list_entries_per_lookup": round(float(stats[2]) / max(float(stats[1]), 1.0), 2),
             "list_entries_per_s": round(float(stats[2]) / (ms / 1e3), 1)}
        if idx == 2:
            # list lengths seen by the starting poses' beads (the workload's "0-80 entries")
            xyz = np.asarray(cfg.ligands[0][0])
            X = np.einsum("bij,nj->bni", euler_to_Q(*poses_np[:20000, :3].T), xyz) + poses_np[:20000, None, 3:]
            g, ng, r = cfg.geom, grid.nb_geom, grid.nb_refine
            v = (X - np.asarray(g.origin)) / g.spacing
            inn = np.all((v >= 0) & (v < np.asarray(g.dim) - 1), axis=2)
            near = np.floor(v * r + 0.5).astype(np.int64)  # nearest list-grid point
            hdr = grid.nb_hdr.cpu().numpy().view(np.uint32)
            vox = (near[..., 0] * ng.dim[1] + near[..., 1]) * ng.dim[2] + near[..., 2]
            cnt = np.where(inn, hdr[np.clip(vox, 0, len(hdr) - 1), 1], 0)
            e["bead_fraction_with_lists"] = round(float((cnt > 0).mean()), 3)
            edges = [0, 1, 6, 11, 21, 41, 81, 1 << 30]
            h = np.histogram(cnt, bins=edges)[0]
            e["list_length_hist"] = {f"{lo}-{hi - 1}" if hi < 1 << 30 else f">={lo}": int(c)
                                     for lo, hi, c in zip(edges[:-1], edges[1:], h)}
            e["list_length_p50_p90_p99"] = [int(x) for x in np.percentile(cnt[cnt > 0], [50, 90, 99])]
            e["list_length_max"] = int(cnt.max())
        res[key] = e
        del grid, wl, scratch
        torch.cuda.empty_cache()
    cfg = synth.make_config(3, seed=0, scale=args.scale)
    grid = A.Grid.build(cfg.rec_xyz, cfg.rec_type, cfg.ff, cfg.geom, cutoff=cfg.cutoff, keep_dense=True,
                        device=device)
    grid.inner.requires_grad_(True)
    grid.outer.requires_grad_(True)
    wl = A.Workload([grid], A.LigandSet(cfg.ligands, device=device), [A.Segment(0, 0, len(cfg.poses[0]))],
                    lanes_per_pose=32)
    P = torch.tensor(cfg.poses[0].astype(np.float32), device=device, requires_grad=True)

    def fwd_bwd():
        P.grad = None
        grid.inner.grad = None
        grid.outer.grad = None
        docking_energy(wl, P, A.EvalOptions(grad_mode="analytic")).backward()

    ms = _timed(fwd_bwd, 10)
    # explicit all-pairs rescoring of the same poses (no grids): 2500 x 24 pairs per pose
    from attract_b200.allpairs import AllPairs

    lig = cfg.ligands[0]
    ap = AllPairs(cfg.rec_xyz, cfg.rec_type, lig[0], lig[2], cfg.ff, device=device)
    Pd = P.detach()
    ms_ap = _timed(lambda: ap.energy(Pd, grad=True), 5)
    n_pairs = len(cfg.rec_type) * len(lig[0]) * wl.n_poses
    res["allpairs"] = {"workload": "explicit all-pairs rescoring with gradient: config-1 receptor (2500 beads) x "
                                   "24-bead ligand x 65536 poses", "ms": round(ms_ap, 3),
                       "value": round(wl.n_poses / ms_ap * 1e3, 1), "unit": "poses/s",
                       "pairs_per_s": round(n_pairs / ms_ap * 1e3, 1)}
    del ap
    # the reference's own protocol (test5.py: 375 adabelief epochs over quaternion poses, SCHEMA
    # stages with gravity) through the drop-in call surface, on 200 000 poses (test5's batch)
    from attract_b200 import reference_api as R
    from attract_b200.poses import random_in_ball

    rng = np.random.default_rng(3)
    nq = max(1000, int(200_000 * args.scale))
    quats = rng.normal(size=(nq, 4))  # uniform rotations: normalised 4-D Gaussians
    quats = (quats / np.linalg.norm(quats, axis=1, keepdims=True)).astype(np.float32)
    trans = random_in_ball(nq, 30.0, rng).astype(np.float32)
    rec_t = np.asarray(cfg.rec_type)
    kw = dict(coor_rec=cfg.rec_xyz, rec_atomtypes=rec_t, coor_lig=lig[0], lig_atomtypes=lig[2], conformers=None,
              lig_atomtype_pos=lig[1], ff=cfg.ff, grid=grid)
    R.minimise_schema(quats[:1000], trans[:1000], **kw, schema=((2, 0.1, True),))  # warm
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    _, _, Ef = R.minimise_schema(quats, trans, **kw, fused=True)
    t1.record()
    torch.cuda.synchronize()
    ms_f = t0.elapsed_time(t1)
    t0.record()
    _, _, Eh = R.minimise_schema(quats, trans, **kw, fused=False)
    t1.record()
    torch.cuda.synchronize()
    ms_h = t0.elapsed_time(t1)
    res["schema"] = {"workload": f"test5 protocol: SCHEMA 375 adabelief epochs, quaternion poses, {nq} poses, "
                                 "config-1 receptor (2500 beads), 24-bead ligand",
                     "fused": {"ms": round(ms_f, 1), "value": round(nq / ms_f * 1e3, 1), "unit": "poses/s"},
                     "per_epoch_launches": {"ms": round(ms_h, 1), "value": round(nq / ms_h * 1e3, 1),
                                            "unit": "poses/s",
                                            "note": "one att_energrad launch per epoch, adabelief in torch ops"},
                     "fused_vs_per_epoch": round(ms_h / ms_f, 2),
                     "median_energy_fused": float(np.median(Ef.cpu().numpy())),
                     "median_energy_per_epoch": float(np.median(Eh.cpu().numpy())),
                     "reference_published": "~3 M structures/hour = 833 poses/s (test5.py:6-7, unspecified "
                                            "hardware; context only)"}
    res["config3"] = {"workload": "differentiation: config-1 receptor, 24-bead ligand, 65536 poses, summed energy, "
                                  "backward to poses and grid energies (analytic mode)",
                      "poses": wl.n_poses, "ms_forward_backward": round(ms, 3),
                      "value": round(wl.n_poses / ms * 1e3, 1), "unit": "poses/s (forward+backward)"}
    del grid, wl
    torch.cuda.empty_cache()
    return res


def serving_run(args, device):
    """Four resident receptors, Poisson arrivals, lognormal pose counts,
    continuous batching in rounds of 50 ADAM steps (200 per request).  Run
    at the workload's arrival rate and, when that overloads the GPU, again at
    60% of the throughput it sustained, where p50/p99 describe a stable queue."""
    import torch

    import attract_b200 as A
    from attract_b200 import synth
    from attract_b200.poses import random_in_ball, random_rotations
    from attract_b200.serve import DockingServer, replay

    ff, recs = synth.serving_mix(seed=0)
    grids = [A.Grid.build(xyz, t, ff, geom, device=device) for xyz, t, R, geom in recs]
    rng = np.random.default_rng(1)
    pool = np.concatenate([random_rotations(400_000, rng), random_in_ball(400_000, 30.0, rng)], 1).astype(np.float32)
    draw = lambda n: pool[(o := int(rng.integers(0, len(pool) - n))):o + n]
    desc = ("4 resident receptors (1500/3000/4500/6000 beads), ligands U{5..60} beads, poses lognormal(median "
            f"10000, sigma 1.0) clipped to [1000, 200000], 200 ADAM steps in rounds of {args.serve_round_steps}; "
            "each round one launch "
            "per launch shape (lanes per pose 8/16/32 and beads per lane by ligand size), rounds pipelined two "
            "deep, a pool of up to 2 M poses in flight")

    def one(rate, seconds):
        srv = DockingServer(grids, steps=200, round_steps=args.serve_round_steps, max_inflight_poses=2_000_000,
                            hbm_budget_bytes=150e9)
        reqs = synth.serving_requests(int(seconds * rate * 1.5) + 10, seed=0, rate=rate)
        st = replay(srv, reqs, duration=seconds, pose_source=draw)
        offered = sum(q["n_poses"] for q in reqs if q["t"] <= seconds) / seconds
        st.update({"arrival_rate_per_s": rate, "offered_poses_per_s": round(offered, 1),
                   "mean_poses_per_request": round(float(np.mean([q["n_poses"] for q in reqs])), 1),
                   "resident_grid_gb": round(srv.grid_bytes / 1e9, 2), "pool_poses": srv.capacity,
                   "gpu_busy": round(st["gpu_s"] / max(st["window_s"], 1e-9), 3)})
        del srv
        return st

    out = {"workload": desc, "window_s_requested": args.serve_seconds,
           "runs": [one(args.serve_rate, args.serve_seconds)]}
    first = out["runs"][0]
    # overloaded: the GPU sustained less than the arrivals offered (requests
    # still in flight when the window closes are not a backlog)
    if first["poses_per_s"] and first["offered_poses_per_s"] > 1.02 * first["poses_per_s"]:
        out["runs"].append(one(round(0.6 * first["poses_per_s"] / first["mean_poses_per_request"], 1),
                               max(20.0, args.serve_seconds / 2)))
    del grids
    torch.cuda.empty_cache()
    return out


def summary(out):
    """The headline figures of the line in a few hundred bytes."""
    r = lambda x, n=1: None if x is None else round(float(x), n)
    sm = {"batched_poses_per_s": out["value"], "e2e_poses_per_s": out["e2e"]["value"],
          "roofline_frac": out["roofline"]["frac"]}
    if "plain" in out:
        sm["plain_poses_per_s"] = out["plain"]["value"]
        sm["batched_vs_plain"] = out["batched_vs_plain"]
    if "cpu_baseline" in out:
        sm["cpu_baseline_poses_per_s"] = r(out["cpu_baseline"]["value"], 2)
    for k, v in out.get("configs", {}).items():
        sm[f"{k}_value"] = v.get("value", (v.get("fused") or {}).get("value"))
        if "bead_fraction_with_lists" in v:
            sm[f"{k}_bead_fraction_with_lists"] = v["bead_fraction_with_lists"]
            sm[f"{k}_list_length_max"] = v["list_length_max"]
    for i, run in enumerate(out.get("serving", {}).get("runs", [])):
        sm[f"serving{i}"] = {"rate": run.get("arrival_rate_per_s"), "poses_per_s": r(run.get("poses_per_s")),
                             "p50_s": r(run.get("p50_s"), 3), "p99_s": r(run.get("p99_s"), 3),
                             "backlog_requests": run.get("backlog_requests")}
    return sm


# --------------------------------------------------------------------------- ours
def run_ours(args):
    import torch

    from attract_b200 import replicas

    R = replicas.init("nccl")  # one process per GPU; replicas, no data-path collective
    rank, world, local, device = R.rank, R.world, R.local, R.device

    import attract_b200 as A
    from attract_b200.autotune import autotune

    A.load_library()
    cfg, grid, ligs, segs, poses_np, order = build(args, device)
    steps = cfg.steps
    wl = A.Workload([grid], ligs, segs)
    poses = torch.tensor(poses_np, device=device)
    tune_ms = {}
    if args.lanes:
        shape = A.LaunchShape(args.lanes, args.threads or 256)
    elif args.no_autotune:
        shape = A.LaunchShape()
    else:
        shape, tune_ms = autotune(wl, poses, use_cache=False)
    wl = wl.with_lanes(shape.lanes_per_pose)

    # statistics launch (untimed): bead evaluations, list lookups, entries
    _, _, _, st = A.minimise(wl, poses, steps, launch=shape, stats=True)
    stats = st.cpu().numpy()
    alg_bytes = algorithmic_bytes(stats)

    plan = A.MinimisePlan(wl, steps, launch=shape)
    plan.pose_in.copy_(poses)
    plan.capture()
    for _ in range(args.warmup):
        plan.replay()
    torch.cuda.synchronize()

    clocks = Clocks(local)
    if rank == 0:
        clocks.start()
    replicas.barrier(R)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        plan.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = replicas.max_over_ranks(R, e0.elapsed_time(e1) / args.steps)
    replicas.barrier(R)
    E = plan.scratch.energy
    status = plan.scratch.status
    n_bad = int((status != 0).sum().item())

    # e2e through the public API: pinned host poses in, energies + poses out
    host_in = torch.from_numpy(poses_np).pin_memory()
    host_E = torch.empty(wl.n_poses, dtype=torch.float32).pin_memory()
    host_P = torch.empty((wl.n_poses, 6), dtype=torch.float32).pin_memory()
    for _ in range(2):
        plan.pose_in.copy_(host_in, non_blocking=True)
        plan.replay()
        host_E.copy_(plan.scratch.energy, non_blocking=True)
        host_P.copy_(plan.pose_out, non_blocking=True)
    torch.cuda.synchronize()
    replicas.barrier(R)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(args.steps):
        plan.pose_in.copy_(host_in, non_blocking=True)
        plan.replay()
        host_E.copy_(plan.scratch.energy, non_blocking=True)
        host_P.copy_(plan.pose_out, non_blocking=True)
    f1.record()
    torch.cuda.synchronize()
    ms_e2e = replicas.max_over_ranks(R, f0.elapsed_time(f1) / args.steps)
    clk = clocks.stop() if rank == 0 else None

    out = None
    if rank == 0:
        n_total = wl.n_poses * world
        value = n_total / (ms / 1e3)
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
        peak = float(peaks.get("hbm_gbs", 6650.0))
        peak_source = ("measured hbm_gbs (MEASURED_PEAKS.json)" if "hbm_gbs" in peaks
                       else "fallback 6650 GB/s (no MEASURED_PEAKS.json on this machine)")
        achieved = alg_bytes / (ms / 1e3) / 1e9
        bead_evals = int(stats[0])
        traffic = traffic_from_profile(bead_evals)
        out = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no public dataset)",
            "config": {"workload": WORKLOAD, "poses_per_step": wl.n_poses, "adam_steps": steps,
                       "evals_per_pose": steps + 1, "l2": "inputs larger than L2 (brick grid "
                       f"{grid.bricks.numel() * 4 / 1e9:.2f} GB, no flush needed)",
                       "launch": {"lanes_per_pose": shape.lanes_per_pose, "block_threads": shape.block_threads},
                       "autotune_ms": tune_ms, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "scale": args.scale},
            "e2e": {"value": round(n_total / (ms_e2e / 1e3), 1), "unit": UNIT,
                    "h2d_bytes_per_step": host_in.numel() * 4, "d2h_bytes_per_step": host_E.numel() * 4 +
                    host_P.numel() * 4},
            "gpu_launches": args.steps * 1,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "algorithmic_bytes_per_launch": alg_bytes, "peak_source": peak_source,
                         "counts": {"brick_reads": int(stats[0]), "list_lookups": int(stats[1]),
                                    "list_entries": int(stats[2])}},
            "clocks": clk,
            "nonfinite_poses": n_bad,
            "median_final_energy": float(E.median().item()),
        }
    if not args.no_plain and rank == 0:
        dt, launches = plain_run(A, grid, cfg, order, poses_np, steps, device)
        out["plain"] = {"value": round(wl.n_poses / dt, 1), "unit": UNIT, "seconds": round(dt, 3),
                        "launches": launches, "note": "one ligand at a time, one energrad launch per step, "
                                                      "ADAM in torch ops"}
        out["batched_vs_plain"] = round(out["value"] / out["plain"]["value"], 2)
    if not args.no_cpu and rank == 0 and world == 1:
        out["cpu_baseline"] = cpu_baseline(cfg, grid, order, args.cpu_poses, steps)
    if rank == 0 and world == 1 and (not args.no_configs or args.serve_seconds > 0):
        del plan, grid, wl
        torch.cuda.empty_cache()
        if not args.no_configs:
            out["configs"] = other_configs(args, device, shape)
        if args.serve_seconds > 0:
            out["serving"] = serving_run(args, device)
    replicas.finish(R)
    if rank == 0:
        out["summary"] = summary(out)  # last: the headline figures survive a truncated tail of the line
        print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------- profiler case
def run_profile_case(args):
    """The minimiser alone on one configuration, launched ``--launches`` times
    (the case the committed ncu summaries capture).  ``--types`` shrinks the
    number of ligand types, and so the grid, to keep captures small; prints
    one JSON line with the mean time of the launches after the first."""
    import torch

    import attract_b200 as A
    from attract_b200 import synth

    A.load_library()
    if args.allpairs:
        return run_profile_allpairs(args)
    cfg = synth.make_config(args.config, seed=0, scale=args.scale, n_types=args.types, clustered=args.clustered)
    steps = cfg.steps if args.adam_steps < 0 else args.adam_steps
    grid = A.Grid.build(cfg.rec_xyz, cfg.rec_type, cfg.ff, cfg.geom, cutoff=cfg.cutoff, nb_refine=args.refine)
    ligs = A.LigandSet(cfg.ligands)
    order = sorted(range(len(cfg.ligands)), key=lambda i: -len(cfg.ligands[i][0]))
    lanes = args.lanes or 32
    wl = A.Workload([grid], ligs, [A.Segment(0, i, len(cfg.poses[i])) for i in order], lanes_per_pose=lanes)
    poses = torch.tensor(np.concatenate([cfg.poses[i] for i in order]).astype(np.float32), device="cuda")
    shape = A.LaunchShape(lanes, args.threads or 128)
    scratch = A.MinimiseScratch(wl.n_poses, wl.device)
    out = torch.empty_like(poses)
    times = []
    for _ in range(args.launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        A.minimise(wl, poses, steps, pose_out=out, launch=shape, scratch=scratch)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    _, _, _, st = A.minimise(wl, poses, steps, launch=shape, stats=True)
    st = st.cpu().numpy().tolist()
    ms = float(np.mean(times[1:])) if len(times) > 1 else times[0]
    print(json.dumps({"config": args.config, "clustered": args.clustered, "scale": args.scale, "types": args.types,
                      "poses": wl.n_poses, "steps": steps, "lanes": lanes, "threads": shape.block_threads, "ms": ms,
                      "poses_per_s": wl.n_poses / ms * 1e3, "stats": st, "brick_gb": grid.bricks.numel() * 4 / 1e9}))


def run_profile_allpairs(args):
    """All-pairs rescoring with gradient of config 3's poses (scaled by
    ``--scale``) on its 2500-bead receptor and 24-bead ligand, ``--launches``
    times; prints the mean time of the launches after the first."""
    import torch

    from attract_b200 import synth
    from attract_b200.allpairs import AllPairs

    cfg = synth.make_config(3, seed=0, scale=args.scale, n_types=args.types)
    xyz, _, lt = cfg.ligands[0]
    ap = AllPairs(cfg.rec_xyz, cfg.rec_type, xyz, lt, cfg.ff)
    P = torch.tensor(cfg.poses[0].astype(np.float32), device="cuda")
    times = []
    for _ in range(args.launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ap.energy(P, grad=True)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.mean(times[1:])) if len(times) > 1 else times[0]
    pairs = len(cfg.rec_type) * len(xyz) * len(P)
    print(json.dumps({"allpairs": True, "poses": len(P), "n_rec": len(cfg.rec_type), "n_lig": len(xyz), "ms": ms,
                      "pairs_per_s": pairs / ms * 1e3, "poses_per_s": len(P) / ms * 1e3}))


# --------------------------------------------------------------------------- reference
def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference_arm

    out = reference_arm.run(args.steps, args.warmup, METRIC, UNIT, WORKLOAD, args.scale)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.profile_case:
        run_profile_case(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
