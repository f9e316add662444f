"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset backs these workloads: receptors, ligands and poses are
generated from ``numpy.random.default_rng(seed)``.

* receptor: beads uniform in a sphere with a minimum separation (random
  sequential addition), types uniform over the force field's types;
* ligand: a random walk (fixed or ranged step length), centred on its centroid;
* poses: uniform rotations (Shoemake), translations uniform in a ball.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .forcefield import ForceField
from .grid import GridGeom
from .poses import random_in_ball, random_rotations

# beads per cubic Angstrom that 2500 beads reach in a 40 A sphere; larger
# receptors grow the sphere so that rejection sampling stays far from jamming
DENSITY_MAX = 2500.0 / (4.0 / 3.0 * np.pi * 40.0 ** 3)


def receptor_beads(n: int, radius: float | None = None, min_sep: float = 3.5, n_types: int = 32, seed: int = 0,
                   density: float | None = None):
    """``n`` beads uniform in a sphere (default radius: 40 A, grown to keep the
    density <= DENSITY_MAX or to ``density`` when given), pairwise >= min_sep."""
    rng = np.random.default_rng(seed)
    if radius is None:
        dens = DENSITY_MAX if density is None else density
        radius = max(40.0 if density is None else 0.0, (n / (dens * 4.0 / 3.0 * np.pi)) ** (1.0 / 3.0))
    cell = min_sep
    cells: dict = {}
    pts = []
    sep2 = min_sep * min_sep
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > 200 * n + 10000:
            raise RuntimeError(f"could not place {n} beads with separation {min_sep} in radius {radius}")
        p = random_in_ball(1, radius, rng)[0]
        key = tuple(np.floor(p / cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in cells.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                        d = p - q
                        if d @ d < sep2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            cells.setdefault(key, []).append(p)
            pts.append(p)
    xyz = np.array(pts)
    types = rng.integers(0, n_types, n)
    return xyz, types, radius


def receptor_beads_clustered(n: int, density: float = 0.01, n_clusters: int = 40, sigma: float = 3.0,
                             min_sep: float = 1.5, n_types: int = 32, seed: int = 0):
    """``n`` beads in dense patches at the same mean density as
    :func:`receptor_beads` with ``density``: ``n_clusters`` Gaussian clusters
    (width ``sigma``) with centres uniform in the sphere and beads pairwise
    >= ``min_sep`` apart, so that neighbour lists within 5 A range from 0
    (between patches) to ~80 entries (patch centres)."""
    rng = np.random.default_rng(seed)
    radius = (n / (density * 4.0 / 3.0 * np.pi)) ** (1.0 / 3.0)
    centres = random_in_ball(n_clusters, max(radius - 2 * sigma, 1.0), rng)
    cell = min_sep
    cells: dict = {}
    pts = []
    sep2 = min_sep * min_sep
    per = np.full(n_clusters, n // n_clusters)
    per[: n - per.sum()] += 1
    for c, m in zip(centres, per):
        placed, tries = 0, 0
        while placed < m:
            tries += 1
            if tries > 2000 * m:
                raise RuntimeError("could not place a cluster's beads")
            p = c + rng.normal(size=3) * sigma * (1.0 + tries / (200.0 * m))  # widen if the core is full
            key = tuple(np.floor(p / cell).astype(int))
            if any(((p - q) @ (p - q)) < sep2 for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
                   for q in cells.get((key[0] + dx, key[1] + dy, key[2] + dz), ())):
                continue
            cells.setdefault(key, []).append(p)
            pts.append(p)
            placed += 1
    xyz = np.array(pts)
    types = rng.integers(0, n_types, n)
    return xyz, types, float(np.linalg.norm(xyz, axis=1).max())


# solvent-accessible surface: bead radius 2.0 A + probe 1.4 A
SAS_RADIUS = 3.4


def surface_points(rec_xyz, n: int, rng, shell: float = 2.0, r_s: float = SAS_RADIUS):
    """``n`` points uniform within ``shell`` of the receptor's solvent-accessible
    surface: the set of points at distance ``r_s`` from their nearest bead
    (the outer envelope and the surfaces of interior cavities alike)."""
    from scipy.spatial import cKDTree

    rec = np.asarray(rec_xyz, np.float64)
    tree = cKDTree(rec)
    lo, hi = rec.min(0) - r_s - shell, rec.max(0) + r_s + shell
    out = []
    got = 0
    while got < n:
        q = rng.uniform(lo, hi, (max(4 * (n - got), 4096), 3))
        d, _ = tree.query(q)
        q = q[np.abs(d - r_s) <= shell]
        out.append(q)
        got += len(q)
    return np.concatenate(out)[:n]


def random_walk(n: int, rng, step=3.8) -> np.ndarray:
    lo, hi = (step, step) if np.isscalar(step) else step
    d = rng.normal(size=(n - 1, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d *= rng.uniform(lo, hi, (n - 1, 1))
    xyz = np.concatenate([np.zeros((1, 3)), np.cumsum(d, 0)])
    return xyz - xyz.mean(0)


@dataclass
class Config:
    name: str
    ff: ForceField
    rec_xyz: np.ndarray
    rec_type: np.ndarray
    rec_radius: float
    geom: GridGeom
    ligands: list                     # (xyz, gtype, ltype)
    poses: list                       # per ligand: [n, 6] float64
    steps: int
    cutoff: float = 10.0
    lr_rot: float = 0.01
    lr_trans: float = 0.05
    extra: dict = field(default_factory=dict)

    @property
    def n_poses(self) -> int:
        return int(sum(len(p) for p in self.poses))


def _poses(n, radius, rng):
    return np.concatenate([random_rotations(n, rng), random_in_ball(n, radius, rng)], 1)


def _ligand(n, rng, n_types, step):
    xyz = random_walk(n, rng, step)
    t = rng.integers(0, n_types, n)
    return xyz, t, t


def make_config(idx: int, seed: int = 0, scale: float = 1.0, n_types: int = 32, clustered: bool = False) -> Config:
    """Config ``idx`` (0..3; the serving mix is :func:`serving_mix`).  ``scale``
    shrinks the pose counts (not the receptor, ligands or steps) for tests.
    ``clustered`` (config 2 only): the receptor's 5000 beads in dense patches at
    the same mean density (:func:`receptor_beads_clustered`), the regime of
    long, ragged neighbour lists."""
    rng = np.random.default_rng(seed)
    ff = ForceField.synthetic(n_types, seed)
    sc = lambda n: max(1, int(round(n * scale)))
    if idx == 0:
        xyz, t, R = receptor_beads(1200, radius=40.0, n_types=n_types, seed=seed + 1)
        ligs = [_ligand(7, rng, n_types, (1.5, 3.8))]
        poses = [_poses(sc(4096), 25.0, rng)]
        steps = 100
    elif idx == 1:
        xyz, t, R = receptor_beads(2500, radius=40.0, n_types=n_types, seed=seed + 1)
        sizes = (18, 21, 24, 26, 28, 30)
        ligs = [_ligand(n, rng, n_types, 3.8) for n in sizes]
        poses = [_poses(sc(100_000), 30.0, rng) for _ in sizes]
        steps = 200
    elif idx == 2:
        if clustered:
            xyz, t, R = receptor_beads_clustered(5000, density=0.01, n_types=n_types, seed=seed + 1)
        else:
            xyz, t, R = receptor_beads(5000, density=0.01, n_types=n_types, seed=seed + 1)
        ligs = [_ligand(40, rng, n_types, 3.8)]
        n = sc(500_000)
        # ligand centroid within 2 A of the receptor's solvent-accessible surface
        poses = [np.concatenate([random_rotations(n, rng), surface_points(xyz, n, rng)], 1)]
        steps = 50
    elif idx == 3:
        xyz, t, R = receptor_beads(2500, radius=40.0, n_types=n_types, seed=seed + 1)
        ligs = [_ligand(24, rng, n_types, 3.8)]
        poses = [_poses(sc(65_536), 30.0, rng)]
        steps = 0
    else:
        raise ValueError(f"config {idx}")
    geom = GridGeom.around((0.0, 0.0, 0.0), R, n_types=n_types)
    return Config(f"config{idx}" + ("-clustered" if clustered and idx == 2 else ""), ff, xyz, t, R, geom, ligs, poses,
                  steps)


def serving_mix(seed: int = 0, n_types: int = 32, sizes=(1500, 3000, 4500, 6000)):
    """The four resident receptors of the serving workload."""
    ff = ForceField.synthetic(n_types, seed)
    recs = []
    for i, n in enumerate(sizes):
        xyz, t, R = receptor_beads(n, n_types=n_types, seed=seed + 10 + i)
        recs.append((xyz, t, R, GridGeom.around((0.0, 0.0, 0.0), R, n_types=n_types)))
    return ff, recs


def serving_requests(n: int, seed: int = 0, n_types: int = 32, rate: float = 200.0, sigma: float = 1.0,
                     median: float = 10_000, clip=(1_000, 200_000), n_receptors: int = 4, radius: float = 30.0):
    """Poisson arrivals; ligand of U{5..60} beads; lognormal pose counts."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for i in range(n):
        nb = int(rng.integers(5, 61))
        npose = int(np.clip(np.round(np.exp(np.log(median) + sigma * rng.normal())), *clip))
        out.append(dict(t=float(t[i]), receptor=int(rng.integers(0, n_receptors)), ligand=_ligand(nb, rng, n_types, 3.8),
                        n_poses=npose, seed=int(rng.integers(0, 2 ** 31))))
    return out
