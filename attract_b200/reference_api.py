"""The reference's energy / gradient call surface, on the B200 kernels.

attract-jax's minimiser (``test5.py``, sjdv1982/attract-jax) scores poses
through ::

    main(rotations, translations, coor_rec, rec_atomtypes, coor_lig,
         lig_atomtypes, conformers, lig_atomtype_pos, ff, grid,
         nb_chunk_thresholds, grid_dim, *, gravity) -> (E_total, E[B])

(test5.py:411-420) and its ``jax.value_and_grad(main, argnums=(0, 1),
has_aux=True)`` (test5.py:429), and minimises with the adabelief SCHEMA loop
of test5.py:436-467.  This module keeps those names, argument meanings and
errors so that a caller can swap the JAX path for the CUDA one:

* ``rotations``: unit quaternions ``[B, 4]`` in scalar-last order (what
  ``Rotation.as_quat()`` returns; an object with ``as_quat()`` is accepted),
  or rotation matrices ``[B, 3, 3]`` for :func:`main`;
* ``translations [B, 3]``; ``conformers [B]`` 0-based indices into
  ``coor_lig [C, N, 3]`` (``coor_lig [N, 3]`` with ``conformers=None`` is one
  conformer);
* ``rec_atomtypes [R]`` / ``lig_atomtypes [N]``: rows / columns of the
  force-field tables; ``lig_atomtype_pos [N]``: potential-grid slot per bead;
* ``ff``: anything with ``rc, ac, ivor`` ``[n_rec_types, n_lig_types]`` (the
  reference's namedtuple, see :func:`make_ff`);
* ``grid``: the namedtuple of ``read_grid(data, read_gradients=True)``
  (read_grid2.py or :mod:`attract_b200.gridfile`) or an :class:`attract_b200.Grid`.

Results are torch tensors on the grid's device.  The rotation gradient is
dE/d(quaternion) through ``Rotation.as_matrix``'s homogeneous quaternion form
(the leaf JAX differentiates), obtained from the kernel's dE/dmat.
``nb_chunk_thresholds`` and ``grid_dim`` tune the reference's JAX chunking and
are accepted and ignored: the kernel walks every list in full.  Argument
errors raise ``AssertionError``, as the reference's asserts do.
"""
from __future__ import annotations

from collections import namedtuple

import numpy as np
import torch

from .engine import EvalOptions, LaunchShape, Segment, Workload, energrad
from .forcefield import ForceField
from .grid import Grid, GridGeom
from .ligand import LigandSet

#: test5.py:14-23, unpacked at test5.py:450 as (epochs, learning rate, gravity)
SCHEMA = ((5, 10.0, True), (10, 5.0, True), (10, 1.0, True), (50, 0.5, True), (100, 0.1, False),
          (100, 0.05, False), (100, 0.02, False))
GRAVITY = 0.1  # test5.py:419

FF = namedtuple("ff", ["rc", "ac", "ivor", "emin", "rmin2"])


def make_ff(rc, ac, ivor) -> FF:
    """The reference's ``ff`` namedtuple (test5.py:132-139): rc, ac, ivor plus
    emin = -27 ac^4 / (256 rc^3) and rmin2 = 4 rc / (3 ac)."""
    rc = np.asarray(rc, np.float64)
    ac = np.asarray(ac, np.float64)
    return FF(rc, ac, np.asarray(ivor, np.float64), -27.0 * ac ** 4 / (256.0 * rc ** 3), 4.0 * rc / (3.0 * ac))


def _np(a):
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def grid_from_reference(grid, coor_rec, rec_atomtypes, ff, device=None) -> Grid:
    """A device :class:`Grid` from the reference's ``Grid`` namedtuple
    (read_grid2.py:16-161, read with gradients) and the receptor it was built for."""
    if isinstance(grid, Grid):
        return grid
    inner = getattr(grid, "inner_potential_grid", None)
    if inner is None or _np(inner).ndim != 5:
        raise AssertionError("the grid must be read with read_gradients=True (test5.py:108)")
    inner = _np(inner)
    outer = getattr(grid, "outer_potential_grid", None)
    geom = GridGeom(tuple(float(v) for v in _np(grid.origin)), float(grid.gridspacing),
                    tuple(int(v) for v in _np(grid.dim)), tuple(int(v) for v in _np(grid.dim2)),
                    int(grid.gridextension), float(grid.plateaudis), int(inner.shape[0]))
    f = ForceField(_np(ff.rc), _np(ff.ac), _np(ff.ivor))
    return Grid.from_dense(geom, _np(coor_rec), _np(rec_atomtypes).astype(np.int64), f, inner=inner,
                           outer=None if outer is None else _np(outer),
                           neighbour_grid=_np(grid.neighbour_grid), nr_neighbours=_np(grid.nr_neighbours),
                           shift_plateau=True, device=device)


class _Prepared:
    """Device-resident inputs for one (grid, receptor, ligand, force field) set."""

    def __init__(self, coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, lig_atomtype_pos, ff, grid, device):
        self.keep = (coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, lig_atomtype_pos, ff, grid)
        self.grid = grid_from_reference(grid, coor_rec, rec_atomtypes, ff, device)
        lig = _np(coor_lig)
        if lig.ndim == 2:
            lig = lig[None]
        if lig.ndim != 3 or lig.shape[-1] != 3:
            raise AssertionError(f"coor_lig must be [C, N, 3] or [N, 3], got {lig.shape}")
        gt = _np(lig_atomtype_pos).astype(np.int64).reshape(-1)
        lt = _np(lig_atomtypes).astype(np.int64).reshape(-1)
        if not (len(gt) == len(lt) == lig.shape[1]):
            raise AssertionError("lig_atomtypes / lig_atomtype_pos do not match the ligand")
        self.n_conf = lig.shape[0]
        self.ligands = LigandSet([(c, gt, lt) for c in lig], device=self.grid.device)
        self.workloads = {}

    def workload(self, n):
        if n not in self.workloads:
            self.workloads = {n: Workload([self.grid], self.ligands, [Segment(0, 0, n)], lanes_per_pose=32)}
        return self.workloads[n]


_CACHE: list = []


def _prepare(coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, lig_atomtype_pos, ff, grid, device=None):
    """The device inputs for these objects, built once and reused while the
    caller passes the same objects (kept alive here so their ids stay valid)."""
    key = tuple(id(o) for o in (coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, lig_atomtype_pos, ff, grid))
    for k, p in _CACHE:
        if k == key:
            return p
    p = _Prepared(coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, lig_atomtype_pos, ff, grid, device)
    _CACHE.insert(0, (key, p))
    del _CACHE[2:]
    return p


def quat_to_matrix(q: torch.Tensor) -> torch.Tensor:
    """``Rotation.as_matrix()`` of scalar-last quaternions, homogeneous form
    (exact for unit quaternions): R = (w^2 - |v|^2) I + 2 v v^T + 2 w [v]x."""
    x, y, z, w = q.unbind(-1)
    return torch.stack([
        torch.stack([x * x - y * y - z * z + w * w, 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        torch.stack([2 * (x * y + z * w), -x * x + y * y - z * z + w * w, 2 * (y * z - x * w)], -1),
        torch.stack([2 * (x * z - y * w), 2 * (y * z + x * w), -x * x - y * y + z * z + w * w], -1)], -2)


def quat_grad(q: torch.Tensor, dEdR: torch.Tensor) -> torch.Tensor:
    """dE/dq from dE/dR through :func:`quat_to_matrix`, written out per component."""
    x, y, z, w = q.unbind(-1)
    G = dEdR
    g00, g01, g02 = G[..., 0, 0], G[..., 0, 1], G[..., 0, 2]
    g10, g11, g12 = G[..., 1, 0], G[..., 1, 1], G[..., 1, 2]
    g20, g21, g22 = G[..., 2, 0], G[..., 2, 1], G[..., 2, 2]
    gx = g00 * x + g01 * y + g02 * z + g10 * y - g11 * x - g12 * w + g20 * z + g21 * w - g22 * x
    gy = -g00 * y + g01 * x + g02 * w + g10 * x + g11 * y + g12 * z - g20 * w + g21 * z - g22 * y
    gz = -g00 * z - g01 * w + g02 * x + g10 * w - g11 * z + g12 * y + g20 * x + g21 * y + g22 * z
    gw = g00 * w - g01 * z + g02 * y + g10 * z + g11 * w - g12 * x - g20 * y + g21 * x + g22 * w
    return 2 * torch.stack([gx, gy, gz, gw], -1)


def _rotations(rotations, device):
    """(quaternions [B,4] or None, matrices [B,3,3]) as float32 device tensors."""
    if hasattr(rotations, "as_quat"):
        rotations = rotations.as_quat()
    r = torch.as_tensor(_np(rotations), dtype=torch.float32, device=device)
    if r.dim() == 2 and r.shape[1] == 4:
        q = r / r.norm(dim=1, keepdim=True)  # Rotation.from_quat normalises
        return q, quat_to_matrix(q)
    return None, r


def check_call(rotations, translations, conformers):
    """The reference's argument checks (test5.py:412), before any device work:
    returns (B, conformer indices or None)."""
    r = rotations.as_quat() if hasattr(rotations, "as_quat") else rotations
    shape = tuple(r.shape) if hasattr(r, "shape") else np.shape(r)
    if not ((len(shape) == 2 and shape[1] == 4) or (len(shape) == 3 and shape[1:] == (3, 3))):
        raise AssertionError(f"rotations must be quaternions [B,4] or matrices [B,3,3], got {shape}")
    B = shape[0]
    tshape = tuple(translations.shape) if hasattr(translations, "shape") else np.shape(translations)
    conf = None if conformers is None else _np(conformers).astype(np.int64).reshape(-1)
    if tshape[:1] != (B,) or (conf is not None and len(conf) != B):
        raise AssertionError("len(rotations) == len(translations) == len(conformers)")
    if tshape != (B, 3):
        raise AssertionError("translations must be [B, 3]")
    if conf is not None and B and conf.min() < 0:
        raise AssertionError("negative conformer index")
    return B, conf


def _evaluate(rotations, translations, coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, conformers,
              lig_atomtype_pos, ff, grid, gravity, grad):
    B, conf = check_call(rotations, translations, conformers)
    prep = _prepare(coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, lig_atomtype_pos, ff, grid)
    dev = prep.grid.device
    q, R = _rotations(rotations, dev)
    t = torch.as_tensor(_np(translations), dtype=torch.float32, device=dev)
    if conf is None:
        if prep.n_conf != 1:
            raise AssertionError("a conformer library needs conformer indices")
        conf = np.zeros(B, np.int64)
    if B and conf.max() >= prep.n_conf:
        raise AssertionError("conformer index outside the conformer library")
    mat = torch.ones((B, 4, 4), dtype=torch.float32, device=dev)  # test5.py:413 starts from ones
    mat[:, :3, :3] = R
    mat[:, 3, :3] = t
    pose_lig = torch.as_tensor(conf.astype(np.int32), device=dev) if prep.n_conf > 1 else None
    opts = EvalOptions(grad_mode="reference", quirk=True, gravity=GRAVITY if gravity else 0.0)
    E, dmat, _ = energrad(prep.workload(B), mat.reshape(B, 16).contiguous(), opts, grad=grad, pose_lig=pose_lig,
                          launch=LaunchShape(32))
    return E, dmat, q


def main(rotations, translations, coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, conformers, lig_atomtype_pos,
         ff, grid, nb_chunk_thresholds=None, grid_dim=None, *, gravity):
    """``(E_total, E [B])`` of the poses (test5.py:411-420)."""
    E, _, _ = _evaluate(rotations, translations, coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, conformers,
                        lig_atomtype_pos, ff, grid, gravity, False)
    return E.sum(), E


def vgrad_main(rotations, translations, coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, conformers,
               lig_atomtype_pos, ff, grid, nb_chunk_thresholds=None, grid_dim=None, *, gravity):
    """``((E_total, E [B]), (dE/dquat [B,4], dE/dtranslation [B,3]))``: the
    reference's ``value_and_grad(main, argnums=(0, 1), has_aux=True)``
    (test5.py:429); rotations must be quaternions."""
    E, dmat, q = _evaluate(rotations, translations, coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, conformers,
                           lig_atomtype_pos, ff, grid, gravity, True)
    if q is None:
        raise AssertionError("vgrad_main differentiates quaternions: pass rotations as [B, 4] quaternions")
    return (E.sum(), E), (quat_grad(q, dmat[:, :3, :3]), dmat[:, 3, :3].contiguous())


class AdaBelief:
    """optax.adabelief(learning_rate) on a list of tensors: b1 0.9, b2 0.999,
    eps 1e-16, eps_root 1e-16; the prediction error is taken against the
    previous first moment, as optax's scale_by_belief does; bias-corrected
    moments; update = -lr * m_hat / (sqrt(s_hat) + eps)."""

    def __init__(self, params, lr, b1=0.9, b2=0.999, eps=1e-16, eps_root=1e-16):
        self.lr, self.b1, self.b2, self.eps, self.eps_root = lr, b1, b2, eps, eps_root
        self.mu = [torch.zeros_like(p) for p in params]
        self.nu = [torch.zeros_like(p) for p in params]
        self.count = 0

    def updates(self, grads):
        self.count += 1
        c1 = 1.0 - self.b1 ** self.count
        c2 = 1.0 - self.b2 ** self.count
        out = []
        for i, g in enumerate(grads):
            err = g - self.mu[i]
            self.mu[i] = self.b1 * self.mu[i] + (1.0 - self.b1) * g
            self.nu[i] = self.b2 * self.nu[i] + (1.0 - self.b2) * err * err + self.eps_root
            out.append(-self.lr * (self.mu[i] / c1) / (torch.sqrt(self.nu[i] / c2) + self.eps))
        return out


def minimise_schema(rotations, translations, coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, conformers,
                    lig_atomtype_pos, ff, grid, schema=SCHEMA, fused=True):
    """The reference's minimisation protocol (test5.py:445-463): per SCHEMA
    stage ``(epochs, learning_rate, gravity)`` a fresh adabelief state over
    (quaternion, translation); each epoch evaluates energies and gradients,
    applies the update and renormalises the quaternion
    (``Rotation.from_quat(rotations.as_quat())``).  Returns ``(quaternions,
    translations, energies)`` where, as in the reference, the energies are
    those of the last evaluation (test5.py:465).  ``fused`` runs the whole
    protocol in one persistent kernel launch (att_minimise_schema); otherwise
    one energy/gradient launch per epoch with the optimiser in torch ops, the
    reference's own dispatch pattern."""
    B, conf = check_call(rotations, translations, conformers)
    prep = _prepare(coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, lig_atomtype_pos, ff, grid)
    q, _ = _rotations(rotations, prep.grid.device)
    if q is None:
        raise AssertionError("minimise_schema takes quaternion rotations")
    t = torch.as_tensor(_np(translations), dtype=torch.float32, device=prep.grid.device)
    if fused:
        from .engine import minimise_schema as _fused

        if conf is None:
            if prep.n_conf != 1:
                raise AssertionError("a conformer library needs conformer indices")
        elif B and conf.max() >= prep.n_conf:
            raise AssertionError("conformer index outside the conformer library")
        qt = torch.zeros((B, 8), dtype=torch.float32, device=prep.grid.device)
        qt[:, :4] = q
        qt[:, 4:7] = t
        pose_lig = (torch.as_tensor(conf.astype(np.int32), device=prep.grid.device)
                    if prep.n_conf > 1 and conf is not None else None)
        out, E, _ = _fused(prep.workload(B), qt, schema, EvalOptions(grad_mode="reference", quirk=True),
                           gravity_weight=GRAVITY, pose_lig=pose_lig, launch=LaunchShape(32))
        return out[:, :4].clone(), out[:, 4:7].clone(), E.clone()
    E = None
    for epochs, lr, gravity in schema:
        opt = AdaBelief([q, t], lr)
        for _ in range(int(epochs)):
            (_, E), (gq, gt) = vgrad_main(q, t, coor_rec, rec_atomtypes, coor_lig, lig_atomtypes, conformers,
                                          lig_atomtype_pos, ff, grid, gravity=gravity)
            uq, ut = opt.updates([gq, gt])
            q = q + uq
            t = t + ut
            q = q / q.norm(dim=1, keepdim=True)
    return q, t, E
