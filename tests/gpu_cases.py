"""Seeded small cases shared by the GPU parity tests (grids, ligands and poses
that exercise the inner grid, the outer grid, the space outside both, the
neighbour lists and the pair-table branches) and the north-star tolerance
check every parity test reports.

The north-star tolerance: per-pose energies within 1e-5 relative (or 1e-4
kcal/mol absolute) of the float64 oracle, gradients within 1e-4 relative
(rotation and translation parts separately, each with a floor of 1e-5 that
only binds for gradients below 0.1).  A pose outside it must lie within a
counted float32 bound (``float32_bounds``):

* arithmetic: 32 u times the sum of the magnitudes of every additive
  component of every term (grid corners; r^-8, r^-6 and plateau parts of the
  pair terms), u = 2^-24 (about 8 rounding steps per term: an approximate
  reciprocal of 1 ulp raised to the 8th power, products and the lane and
  shuffle-tree sums);
* inputs: the float32 bead positions, off by up to delta = 8 u (|x| + |X| +
  |X - o|) (rotation from float32 sines, the product with the ligand frame,
  the translation and the grid-frame shift): the spread of each bead's
  float64 energy and gradient over +-2 delta along each axis, which covers
  the slope and any jump within reach (a cell face of the analytic gradient,
  the energy cap, the inner/outer grid boundary);
* the trilinear quirk: the reference's floor/ceil weights give 0 for a bead
  whose voxel coordinate is an exact integer; a float32 coordinate within
  reach of an integer (about one bead in 30 000) may land on it and lose
  its whole grid term, which the float64 coordinate does not.
"""
from __future__ import annotations

import numpy as np

import attract_oracle as O

U = 2.0 ** -24
NS_E_REL, NS_E_ABS, NS_G_REL = 1e-5, 1e-4, 1e-4
G_FLOOR = 1e-5  # kcal/mol/A (/rad): only binds for gradients below 0.1


def small_case(seed=0, n_types=4, n_rtypes=3, n_rec=60, n_lig_beads=9, n_poses=64, cap=True, ivor_mix=False,
               plateau=3.5, spacing=1.0, with_outer=True, with_grid=True, with_nb=True):
    rng = np.random.default_rng(seed)
    dim = np.array([14, 13, 12])
    ext = 4
    dim2 = np.array([11, 10, 10])
    origin = np.array([-6.5, -6.0, -5.5])
    geom = dict(origin=origin, spacing=spacing, dim=dim, dim2=dim2, extension=ext, plateau=plateau)
    sigma = rng.uniform(2.0, 3.0, (n_rtypes, n_types))
    eps = rng.uniform(0.1, 2.0, (n_rtypes, n_types))
    rc, ac = eps * sigma ** 8, eps * sigma ** 6
    ivor = np.ones_like(rc)
    if ivor_mix:
        ivor = np.where(rng.random(rc.shape) < 0.5, -1.0, 1.0)
    rcap2 = (0.6 * sigma) ** 2 if cap else np.zeros_like(sigma)
    box_lo = origin + 1.0
    box_hi = origin + (dim - 2) * spacing
    rec = rng.uniform(box_lo, box_hi, (n_rec, 3))
    rtype = rng.integers(0, n_rtypes, n_rec)
    pair = O.pair_table(rc, ac, ivor, plateau, shift_plateau=with_grid, rcap2=rcap2)
    G = dict(geom=geom, rec=rec, rtype=rtype, pair=pair)
    if with_grid:
        G["inner"] = rng.normal(size=(n_types, *dim, 4))
        if with_outer:
            G["outer"] = rng.normal(size=(n_types, *dim2, 4))
    if with_nb:
        G["nb_hdr"], G["nb_list"] = O.build_nbgrid(rec, geom, plateau + spacing * np.sqrt(3) / 2 + 0.05)
    lig = O.transform(np.zeros(6), rng.normal(size=(n_lig_beads, 3)) * 1.6)
    lig -= lig.mean(0)
    gt = rng.integers(0, n_types, n_lig_beads)
    lt = rng.integers(0, n_types, n_lig_beads)
    ang = rng.uniform(-np.pi, np.pi, (n_poses, 3))
    centre = origin + (dim - 1) * spacing / 2
    # most poses inside the inner grid, some straddling into the outer grid or beyond
    r = np.where(rng.random(n_poses) < 0.75, rng.uniform(0, 4.0, n_poses), rng.uniform(5.0, 14.0, n_poses))
    d = rng.normal(size=(n_poses, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = centre + d * r[:, None]
    poses = np.concatenate([ang, t], 1)
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)
    G["rec"] = f32(G["rec"])
    for k in ("inner", "outer"):
        if k in G:
            G[k] = f32(G[k])
    lig, poses = f32(lig), f32(poses)
    return dict(G=G, lig=lig, gt=gt, lt=lt, poses=poses, rc=rc, ac=ac, ivor=ivor, rcap2=rcap2,
                n_types=n_types, n_rtypes=n_rtypes, with_grid=with_grid)


def to_device_grid(case, device="cuda"):
    """The case's grid as an attract_b200 Grid (same arrays as the oracle sees)."""
    from attract_b200 import ForceField, Grid, GridGeom

    G = case["G"]
    g = G["geom"]
    geom = GridGeom(tuple(g["origin"]), g["spacing"], tuple(g["dim"]), tuple(g["dim2"]), g["extension"],
                    g["plateau"], case["n_types"])
    ff = ForceField(case["rc"], case["ac"], case["ivor"], case["rcap2"])
    return Grid.from_dense(geom, G["rec"], G["rtype"], ff, inner=G.get("inner"), outer=G.get("outer"),
                           nb_hdr=G.get("nb_hdr"), nb_list=G.get("nb_list"), shift_plateau=case["with_grid"],
                           keep_dense=True, device=device)


def oracle_scales(case, poses, mode="reference", quirk=True, position_term=False):
    """Per-pose magnitude scales for float32 tolerances: the sum over every
    grid corner and pair term of |energy term|, and of |gradient term| * (1 + |r_b|)
    (float32 summation error is bounded relative to these, not to a total
    in which large terms cancel).  ``position_term`` adds the float32 rounding
    of the bead positions, |dE/dx| |x| ~1e-7, which dominates for steep
    uncapped clashes."""
    G = case["G"]
    X = O.transform(poses, case["lig"])
    absG = dict(G)
    for k in ("inner", "outer"):
        if k in G:
            absG[k] = np.abs(G[k])
    Eg, gg = O.grid_energrad(X, case["gt"], G["geom"], absG.get("inner"), absG.get("outer"), quirk, "reference")
    En, gn = O.nb_energrad(X, case["lt"], G["geom"], G.get("nb_hdr"), G.get("nb_list"), G["rec"], G["rtype"],
                           G["pair"], mode, absolute=True)
    if mode == "analytic":  # the analytic grid gradient is bounded by |E corners| / spacing
        gg = np.repeat(Eg[..., None], 3, -1) * 2.0 / G["geom"]["spacing"]
    r = X - poses[:, None, 3:6]
    gabs = (np.abs(gg) + gn).sum(-1)
    es = (Eg + En).sum(1)
    if position_term:
        es = es + 0.2 * (gabs * (1 + np.linalg.norm(X, axis=2))).sum(1)
    gs = (gabs * (1 + np.linalg.norm(r, axis=2))).sum(1)
    return es, gs


def float32_bounds(poses, lig, gt, lt, G, mode):
    """Per-pose (energy, rotation-gradient, translation-gradient) float32 bounds."""
    X = O.transform(poses, lig)                                     # [B, N, 3]
    t = poses[:, None, 3:6]
    ab = lambda a: None if a is None else np.abs(a)
    Eg, gg = O.grid_energrad(X, gt, G["geom"], ab(G.get("inner")), ab(G.get("outer")), True, "reference")
    En, gn = O.nb_energrad(X, lt, G["geom"], G.get("nb_hdr"), G.get("nb_list"), G["rec"], G["rtype"], G["pair"],
                           mode, absolute=True)
    if mode == "analytic":
        gg = np.repeat(Eg[..., None], 3, -1) * 2.0 / G["geom"]["spacing"]
    S_e = Eg + En                                                   # [B, N]
    S_g = np.linalg.norm(np.abs(gg) + gn, axis=-1)                  # [B, N]
    o = np.asarray(G["geom"]["origin"])
    delta = 8 * U * (np.linalg.norm(lig, axis=-1)[None] + np.linalg.norm(X, axis=-1) + np.linalg.norm(X - o, axis=-1))
    # the bead terms' spread over the float32 position uncertainty, probed
    # along each axis at +-2 delta: the slope in smooth regions, and any jump
    # within reach (an analytic-gradient cell face, the energy cap, the
    # inner/outer grid boundary) that float32 positions may land across
    _, gb = O.bead_energrad(X, gt, lt, G, mode)
    sE = np.zeros(X.shape[:2])
    sG = np.zeros(X.shape[:2])
    for k in range(3):
        d = np.zeros(X.shape)
        d[..., k] = 2 * delta
        Ep, gp = O.bead_energrad(X + d, gt, lt, G, mode)
        Em, gm = O.bead_energrad(X - d, gt, lt, G, mode)
        sE = np.maximum(sE, np.abs(Ep - Em))
        sG = np.maximum(sG, np.linalg.norm(gp - gm, axis=-1))
    # the reference's floor/ceil weights zero a bead whose voxel coordinate is
    # an exact integer (test5.py:256-259): a float32 coordinate within reach
    # of an integer may land on it, which removes the bead's whole grid term
    g = G["geom"]
    v = (X - o) / g["spacing"]
    inn = np.all((v >= 0) & (v < np.asarray(g["dim"]) - 1), axis=-1)
    vo = (v + g["extension"]) / 2.0
    vv = np.where(inn[..., None], v, vo)
    dv = np.where(inn, 1.0, 0.5)[..., None] * (2 * delta[..., None] / g["spacing"] + 8 * U * np.abs(vv))
    on_int = np.any(np.abs(vv - np.round(vv)) <= dv, axis=-1)
    qE = np.where(on_int, Eg, 0.0)
    qG = np.where(on_int, np.linalg.norm(np.abs(gg), axis=-1), 0.0)
    sE = sE + qE
    sG = sG + qG
    arm = 1.0 + np.linalg.norm(X - t, axis=-1)
    gnorm = np.linalg.norm(gb, axis=-1)
    bE = 32 * U * S_e.sum(1) + sE.sum(1)
    bT = 32 * U * S_g.sum(1) + sG.sum(1)
    bR = 2.0 * (32 * U * (S_g * arm).sum(1) + (sG * arm + gnorm * delta).sum(1))
    return bE, bR, bT


def north_star_report(name, E, G, Eo, Go, bounds):
    """Fractions within the north-star tolerance; asserts the rest lie within
    the float32 bounds.  Returns the report dict (also printed)."""
    bE, bR, bT = bounds
    dE = np.abs(E - Eo)
    tolE = np.maximum(NS_E_REL * np.abs(Eo), NS_E_ABS)
    inE = dE <= tolE
    out = {"poses": len(E), "energy_within_1e-5": float(inE.mean())}
    ok = inE | (dE <= bE)
    worst = {"energy": float((dE / np.maximum(tolE, bE)).max())}
    if G is not None:  # rotation part: every column but the last three (Euler angles or the 3x3 block)
        G, Go = G.reshape(len(G), -1), Go.reshape(len(Go), -1)
        dR = np.linalg.norm(G[:, :-3] - Go[:, :-3], axis=1)
        dT = np.linalg.norm(G[:, -3:] - Go[:, -3:], axis=1)
        tolR = NS_G_REL * np.linalg.norm(Go[:, :-3], axis=1) + G_FLOOR
        tolT = NS_G_REL * np.linalg.norm(Go[:, -3:], axis=1) + G_FLOOR
        inG = (dR <= tolR) & (dT <= tolT)
        out["gradient_within_1e-4"] = float(inG.mean())
        out["both_within"] = float((inE & inG).mean())
        ok &= ((dR <= tolR) | (dR <= bR)) & ((dT <= tolT) | (dT <= bT))
        worst["rotation"] = float((dR / np.maximum(tolR, bR)).max())
        worst["translation"] = float((dT / np.maximum(tolT, bT)).max())
        out["outside_explained_by_float32_bound"] = int(((~(inE & inG)) & ok).sum())
    else:
        out["outside_explained_by_float32_bound"] = int(((~inE) & ok).sum())
    out["max_error_over_allowed"] = worst
    out["unexplained"] = int((~ok).sum())
    print(f"\n[north-star] {name}: {out}")
    assert out["unexplained"] == 0, (name, out, np.flatnonzero(~ok)[:10])
    return out
