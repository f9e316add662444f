"""Parity at the benchmark workloads' own shapes, through the C ABI.

The grids here are the ones ``bench.py`` times: the synthetic receptors of
the scoring configurations (1200 / 2500 / 5000 beads), 32 types, potentials
built on the GPU, neighbour lists on the inner grid refined x4 with 32-byte
inline records and CSR overflow.  Poses are samples of each configuration's
own poses.  The oracle (float64 NumPy restatement of test5.py:255-429, the
minimiser of test4.py:440-455) evaluates the same float32 inputs: the
kernel's grids, lists (device order), receptor, ligand and poses.

Every test prints the north-star metric directly -- the fraction of poses
whose energy is within 1e-5 relative (or 1e-4 kcal/mol absolute) of the
float64 oracle and whose gradient is within 1e-4 relative -- and asserts that
every pose outside it lies within the counted float32 bound of
``gpu_cases.float32_bounds``.
"""
import numpy as np
import pytest
import torch

import attract_oracle as O
from gpu_cases import G_FLOOR, NS_G_REL, float32_bounds, north_star_report

pytestmark = pytest.mark.gpu


def _A():
    import attract_b200 as A

    A.load_library()
    return A


# ----------------------------------------------------------------------------- workloads
_CACHE = {}


def _config(idx):
    """(cfg, grid, oracle grid dict) of configuration ``idx`` (``"2c"``: config
    2 with the clustered receptor; ``"2c32"``: the same with 32-byte records,
    so that most long lists continue in the CSR overflow), built once."""
    if idx in _CACHE:
        return _CACHE[idx]
    for k in list(_CACHE):  # one configuration's grids resident at a time
        del _CACHE[k]
    _ORACLE.clear()
    torch.cuda.empty_cache()
    A = _A()
    from attract_b200 import synth

    clustered = idx in ("2c", "2c32")
    cfg = synth.make_config(2 if clustered else idx, seed=0, clustered=clustered)
    grid = A.Grid.build(cfg.rec_xyz, cfg.rec_type, cfg.ff, cfg.geom, cutoff=cfg.cutoff, keep_dense=True)
    if idx == "2c32":
        grid._pack_records(32)
        grid._att = None
    _CACHE[idx] = (cfg, grid, oracle_grid(grid, cfg.ff))
    return _CACHE[idx]


def oracle_grid(grid, ff):
    """The device grid as the oracle's dict: dense float32 potentials, the
    lists as the kernels read them (receptor beads in device order), the
    float32 receptor, and the geometry rounded to float32 as the device holds it."""
    rec = grid.rec.cpu().numpy()[: grid.n_rec]
    g = grid.geom.as_dict()
    g["origin"] = np.asarray(g["origin"], np.float32).astype(np.float64)
    g["spacing"] = float(np.float32(g["spacing"]))
    g["nb_refine"] = grid.nb_refine
    return dict(geom=g, inner=grid.inner.cpu().numpy(), outer=grid.outer.cpu().numpy(),
                nb_hdr=grid.nb_hdr.cpu().numpy().view(np.uint32), nb_list=grid.nb_list.cpu().numpy().view(np.uint16),
                rec=rec[:, :3].astype(np.float64), rtype=rec[:, 3].copy().view(np.int32).astype(np.int64),
                pair=O.pair_table(ff.rc, ff.ac, ff.ivor, grid.geom.plateau, True, ff.rcap2))


def _f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def sample(cfg, per_lig):
    """The first ``per_lig`` poses of every ligand: [(ligand index, poses)]."""
    return [(i, _f32(p[:per_lig])) for i, p in enumerate(cfg.poses)]


# ----------------------------------------------------------------------------- energrad
_ORACLE = {}
# grouped by configuration, so that each configuration's grids are built once
ENERGRAD_CASES = [(idx, n, lanes, mode) for idx, n, shapes in ((0, 4096, (8, 32)), (1, 256, (32, 8)),
                                                                (2, 2048, (32, 16)), ("2c", 2048, (32,)),
                                                                ("2c32", 2048, (32,)))
                  for mode in ("reference", "analytic") for lanes in shapes]


@pytest.mark.parametrize("idx,per_lig,lanes,mode", ENERGRAD_CASES)
def test_config_energrad_vs_fp64(idx, per_lig, lanes, mode):
    """One energy + gradient evaluation of sampled configuration poses (config
    0: all 4096; config 1: 256 per fragment; config 2: 2048 surface poses,
    with the uniform and the clustered receptor, whose lists of up to ~80
    entries take 128-byte records -- and, repacked into 32-byte records, run
    far past the inline entries into the CSR overflow) against the float64
    oracle, at one or two launch shapes."""
    A = _A()
    cfg, grid, G = _config(idx)
    parts = sample(cfg, per_lig)
    ligs = A.LigandSet(cfg.ligands)
    wl = A.Workload([grid], ligs, [A.Segment(0, i, len(p)) for i, p in parts], lanes_per_pose=lanes)
    P = torch.tensor(np.concatenate([p for _, p in parts]), dtype=torch.float32, device="cuda")
    E, Gr, S = A.energrad(wl, P, A.EvalOptions(grad_mode=mode))
    E, Gr, S = E.cpu().numpy(), Gr.cpu().numpy(), S.cpu().numpy()
    assert np.all(S == 0)
    key = (idx, per_lig, mode)
    if key not in _ORACLE:  # the oracle side does not depend on the launch shape
        res = []
        for i, p in parts:
            xyz, gt, lt = cfg.ligands[i]
            lig = _f32(xyz)
            res.append(O.energrad(p, lig, gt, lt, G, mode=mode) + float32_bounds(p, lig, gt, lt, G, mode))
        _ORACLE[key] = [np.concatenate([r[k] for r in res]) for k in range(5)]
    Eo, Go, bE, bR, bT = _ORACLE[key]
    north_star_report(f"config {idx}, {mode} gradient, {lanes} lanes", E, Gr, Eo, Go, (bE, bR, bT))


# ----------------------------------------------------------------------------- minimisation
def _rank_metrics(E, Eref):
    from scipy.stats import spearmanr

    n = len(E)
    out = {"spearman": float(spearmanr(E, Eref).correlation)}
    for frac in (0.01, 0.05):
        k = max(1, int(round(frac * n)))
        a = set(np.argsort(E)[:k].tolist())
        b = set(np.argsort(Eref)[:k].tolist())
        out[f"top{int(frac * 100)}pct_overlap"] = len(a & b) / k
    out["final_energy_within_1e-3_rel"] = float(np.mean(np.abs(E - Eref) <= 1e-3 * np.maximum(np.abs(Eref), 1.0)))
    return out


MIN_CASES = [(0, 1024, 8), (1, 64, 32), (2, 256, 32), ("2c", 256, 32)]


@pytest.mark.parametrize("idx,per_lig,lanes", MIN_CASES)
def test_config_minimisation_ranking_vs_fp64(idx, per_lig, lanes):
    """Full-length fused ADAM runs (config 0: 100 steps, config 1: 200,
    config 2: 50; lr 0.01 rad / 0.05 A) on pose samples against the float64
    oracle's minimiser.  Reported: Spearman correlation and top-1 % / top-5 %
    overlap of the final energies, for the kernel and -- as the floor any
    float32 run has -- for the oracle's own float32-arithmetic run."""
    A = _A()
    cfg, grid, G = _config(idx)
    parts = sample(cfg, per_lig)
    ligs = A.LigandSet(cfg.ligands)
    wl = A.Workload([grid], ligs, [A.Segment(0, i, len(p)) for i, p in parts], lanes_per_pose=lanes)
    P = torch.tensor(np.concatenate([p for _, p in parts]), dtype=torch.float32, device="cuda")
    out, E, S, _ = A.minimise(wl, P, cfg.steps)
    E = E.cpu().numpy()
    assert np.all(np.isfinite(E))
    E64, E32 = [], []
    for i, p in parts:
        xyz, gt, lt = cfg.ligands[i]
        lig = _f32(xyz)
        E64.append(O.minimise(p, lig, gt, lt, G, cfg.steps, cfg.lr_rot, cfg.lr_trans)[1])
        E32.append(O.minimise(p, lig, gt, lt, G, cfg.steps, cfg.lr_rot, cfg.lr_trans, dtype=np.float32)[1])
    E64, E32 = np.concatenate(E64), np.concatenate(E32)
    gpu = _rank_metrics(E, E64)
    f32 = _rank_metrics(E32, E64)
    print(f"\n[ranking] config {idx} ({len(E)} poses, {cfg.steps} ADAM steps): kernel vs float64 {gpu}; "
          f"oracle float32 vs float64 {f32}")
    assert gpu["spearman"] >= min(0.98, f32["spearman"] - 0.01), (gpu, f32)
    assert gpu["top5pct_overlap"] >= min(0.8, f32["top5pct_overlap"] - 0.1), (gpu, f32)
    # the energy reported is the energy of the pose returned
    Ef, _, _ = A.energrad(wl, out.contiguous())
    assert np.allclose(Ef.cpu().numpy(), E, rtol=1e-6, atol=1e-5)


# ----------------------------------------------------------------------------- differentiation
def test_config3_finite_differences_poses_and_voxels():
    """Differentiation workload (config-1 receptor, 24-bead ligand, 65 536
    poses): the summed energy's backward -- dE/d(pose) and dE/d(grid energy
    value) -- against float64 central finite differences (h = 1e-4) of the
    oracle on 256 sampled poses and 256 sampled voxels, and the reference-mode
    backward against the oracle's reference (analytic JAX-style) gradient."""
    A = _A()
    from attract_b200.autograd import docking_energy

    cfg, grid, G = _config(3)
    xyz, gt, lt = cfg.ligands[0]
    lig = _f32(xyz)
    poses = _f32(cfg.poses[0])
    wl = A.Workload([grid], A.LigandSet(cfg.ligands), [A.Segment(0, 0, len(poses))], lanes_per_pose=32)
    grid.inner.requires_grad_(True)
    grid.outer.requires_grad_(True)
    P = torch.tensor(poses, dtype=torch.float32, device="cuda", requires_grad=True)
    docking_energy(wl, P, A.EvalOptions(grad_mode="analytic")).backward()
    gpose = P.grad.cpu().numpy().astype(np.float64)
    din = grid.inner.grad.cpu().numpy()
    grid.inner.requires_grad_(False)
    grid.outer.requires_grad_(False)
    rng = np.random.default_rng(7)
    pick = rng.choice(len(poses), 256, replace=False)
    sp = poses[pick]
    # --- poses: central differences of the float64 oracle energy
    h = 1e-4
    fd = np.zeros((256, 6))
    for k in range(6):
        pp, pm = sp.copy(), sp.copy()
        pp[:, k] += h
        pm[:, k] -= h
        fd[:, k] = (O.energrad(pp, lig, gt, lt, G, mode="analytic")[0] -
                    O.energrad(pm, lig, gt, lt, G, mode="analytic")[0]) / (2 * h)
    _, ga = O.energrad(sp, lig, gt, lt, G, mode="analytic")
    g = gpose[pick]
    tol = lambda ref: NS_G_REL * np.linalg.norm(ref, axis=1)[:, None] + G_FLOOR
    b = float32_bounds(sp, lig, gt, lt, G, "analytic")
    # (1) the kernel against the float64 analytic gradient: north-star report
    north_star_report("config 3 backward dE/dpose vs float64 analytic", np.zeros(256), g, np.zeros(256), ga,
                      (np.zeros(256), b[1], b[2]))
    # (2) finite differences: where no bead crosses a cell face or the energy
    # cap within +-h, FD equals the analytic float64 gradient to its truncation error
    smooth = np.all(np.abs(fd - ga) <= 1e-3 * (np.abs(ga).max(1, keepdims=True) + 1.0), axis=1)
    agree = np.all(np.abs(g - fd) <= np.maximum(tol(fd), 1e-3 * (np.abs(fd).max(1, keepdims=True) + 1.0)), axis=1)
    rep = {"poses": 256, "fd_smooth": float(smooth.mean()), "kernel_vs_fd_within": float(agree[smooth].mean())}
    print(f"\n[fd poses] {rep}")
    assert smooth.mean() > 0.85 and agree[smooth].mean() >= 0.99, rep
    # (3) reference-mode backward = the oracle's reference gradient (test5.py:429 semantics)
    Pr = torch.tensor(sp, dtype=torch.float32, device="cuda", requires_grad=True)
    wl_s = A.Workload([grid], A.LigandSet(cfg.ligands), [A.Segment(0, 0, 256)], lanes_per_pose=32)
    docking_energy(wl_s, Pr, A.EvalOptions(grad_mode="reference")).backward()
    Eo, gr = O.energrad(sp, lig, gt, lt, G, mode="reference")
    br = float32_bounds(sp, lig, gt, lt, G, "reference")
    north_star_report("config 3 backward dE/dpose vs float64 reference gradient", np.zeros(256),
                      Pr.grad.cpu().numpy().astype(np.float64), np.zeros(256), gr, (np.zeros(256), br[1], br[2]))
    # --- voxels: E is linear in each grid energy value, so the central
    # difference equals the sum of that voxel's trilinear weights over every
    # bead of every pose that reads it; evaluated on those poses only
    X = O.transform(poses, lig)
    g0 = G["geom"]
    v = (X - np.asarray(g0["origin"])) / g0["spacing"]
    inn = np.all((v >= 0) & (v < np.asarray(g0["dim"]) - 1), axis=2)
    base = np.floor(v).astype(np.int64)
    touched = np.argwhere(din[..., 0] != 0)
    vox = touched[rng.choice(len(touched), 256, replace=False)]
    inner64 = G["inner"].astype(np.float64)
    G64 = dict(G, inner=inner64)
    worst = worst_bound = 0.0
    for t_, x_, y_, z_ in vox:
        near = inn & (gt[None, :] == t_) & np.all(
            (base >= np.array([x_, y_, z_]) - 1) & (base <= np.array([x_, y_, z_])), axis=2)
        rows = np.flatnonzero(near.any(1))
        assert len(rows), (t_, x_, y_, z_)
        old = inner64[t_, x_, y_, z_, 0]
        inner64[t_, x_, y_, z_, 0] = old + h
        Ep = O.energrad(poses[rows], lig, gt, lt, G64, mode="analytic")[0].sum()
        inner64[t_, x_, y_, z_, 0] = old - h
        Em = O.energrad(poses[rows], lig, gt, lt, G64, mode="analytic")[0].sum()
        inner64[t_, x_, y_, z_, 0] = old
        fdv = (Ep - Em) / (2 * h)
        # float32 bound of the kernel's value: it adds the voxel's n weights one
        # by one (atomics: n u relative), each weight a product of fractional
        # voxel coordinates of a float32 bead position (off by up to 2 delta /
        # spacing per axis, 3 axes: the bound of gpu_cases.float32_bounds)
        n_terms = int(near.sum())
        Xn = X[near]
        delta = 8 * 2.0 ** -24 * (np.linalg.norm(lig, axis=1)[np.nonzero(near)[1]] + np.linalg.norm(Xn, axis=1) +
                                  np.linalg.norm(Xn - np.asarray(g0["origin"]), axis=1))
        bound = 2 * n_terms * 2.0 ** -24 * abs(fdv) + float((3 * 2 * delta / g0["spacing"]).sum())
        err = abs(din[t_, x_, y_, z_, 0] - fdv)
        worst = max(worst, err / max(1.0, abs(fdv)))
        worst_bound = max(worst_bound, err / max(1e-5 * max(1.0, abs(fdv)), bound))
    print(f"\n[fd voxels] 256 voxels, max relative error {worst:.2e} "
          f"({worst_bound:.2f} of max(1e-5 relative, float32 bound))")
    assert worst_bound <= 1.0, (worst, worst_bound)
