"""CPU oracle for the ATTRACT grid/nbgrid scoring-and-minimisation path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: the parity tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it.
The product path (``attract_b200``) never imports it and has no CPU fallback.

It restates, in NumPy (float64 by default, float32 on request), the algorithm of
the reference's JAX minimiser ``test5.py`` (sjdv1982/attract-jax), function by
function; every function cites the reference lines it follows.  The reference
itself cannot run here (no jax/optax), so the restatement is pinned against the
reference's own golden outputs instead (``tests/golden``):

* ``nonbon``                     -> ``energy-init/score.out`` (ATTRACT, 296 distances)
* pose application + all pairs   -> ``mono-leu/minim-sorted.score`` (ATTRACT energies)
* Euler convention               -> ``mono-leu/minim-sorted.dat`` vs ``minim-sorted.npy``
* nb pair term, plain            -> ``test-nb-energrad.out`` (JAX) and
                                    ``mono-leu/minim-sorted-nbgrid.score`` (ATTRACT
                                    energies + Euler/translation gradients)
* nb pair term, plateau-shifted  -> ``test-nb-energrad-plateau.out`` (JAX, the
  (test5 semantics)                 custom-JVP plateau correction)

The trilinear potential-grid term (test5.py:255-311) has no golden vector that
can be recomputed here (the ATTRACT ``.grid`` files are absent from the
reference): that part is a restatement only ("grid term: parity unpinned").

Conventions
-----------
pose  = (phi, psi, theta, tx, ty, tz), the ATTRACT ``.dat`` order.  The
reference's row-vector matrix is ``mat[:3,:3] = Rz(theta) Ry(-psi) Rz(-phi)``
(scipy ``from_euler('zyz', [-phi, -psi, theta])``), ``mat[3,:3] = t``, and a
ligand bead moves to ``[x, 1] @ mat`` (test5.py:315-317).  In column form the
rotation applied is ``Q = mat[:3,:3].T = Rz(phi) Ry(psi) Rz(-theta)``.

Pair table ``pair[l, r, k]`` (ligand type l, receptor type r), k =
``rc, ac, emin, rmin2, ivor, eplat, gplat, rcap2`` -- the ``ff`` namedtuple of
test5.py:122-140 plus the plateau tables of test5.py:208-211 and an optional
energy cap (``rcap2`` = 0 reproduces the reference exactly).
"""
from __future__ import annotations

import numpy as np

NB_EMPTY = 65535  # empty neighbour slot, test5.py:240 / read_grid2.py:118

PAIR_FIELDS = ("rc", "ac", "emin", "rmin2", "ivor", "eplat", "gplat", "rcap2")


# --------------------------------------------------------------------------
# force field (test5.py:122-140; attract-original/convert-attract-par.py:1-22)
# --------------------------------------------------------------------------
def ff_from_attract_par(text: str):
    """Parse an ATTRACT ``attract.par`` file into (rc, ac, ivor) [ntypes, ntypes].

    Follows convert-attract-par.py:1-22: header ``potshape ntypes``, then three
    ntypes x ntypes blocks rbc, abc, ipon; rc = abc*rbc**8, ac = abc*rbc**6.
    """
    lines = text.splitlines()
    header = [int(x) for x in lines[0].split()]
    potshape, ntypes = header[0], header[1]
    assert potshape == 8
    vals = np.array(" ".join(lines[1:]).split(), dtype=np.float64)
    par = vals[: 3 * ntypes * ntypes].reshape(3, ntypes, ntypes)
    rbc, abc, ipon = par[0], par[1], par[2].astype(int)
    rc = abc * rbc ** potshape
    ac = abc * rbc ** 6
    return rc, ac, ipon.astype(np.float64)


def nonbon(dsq, rc, ac, emin, rmin2, ivor, rcap2=0.0):
    """ATTRACT 8-6 pair energy of a squared distance (test5.py:186-202).

    ``rcap2`` > 0 caps the energy at ``nonbon(rcap2)`` below that squared
    distance (an extension; 0 reproduces the reference).
    """
    d = np.maximum(dsq, rcap2)
    rr2 = 1.0 / d
    rr23 = rr2 * rr2 * rr2
    vlj = (rc * rr2 - ac) * rr23
    return np.where(d < rmin2, vlj + (ivor - 1.0) * emin, ivor * vlj)


def dnonbon_ddsq(dsq, rc, ac, emin, rmin2, ivor, rcap2=0.0):
    """d nonbon / d dsq -- ``grad_nonbon`` of test5.py:204 (jax.grad w.r.t. dsq)."""
    d = np.maximum(dsq, rcap2)
    rr2 = 1.0 / d
    dv = rr2 ** 4 * (3.0 * ac - 4.0 * rc * rr2)
    g = np.where(d < rmin2, dv, ivor * dv)
    return np.where(dsq < rcap2, 0.0, g)


def pair_table(rc, ac, ivor, plateau, shift_plateau=True, rcap2=None):
    """Per-pair parameter table ``[n_ltypes, n_rtypes, 8]``.

    rc/ac/ivor are given receptor-major ``[n_rtypes, n_ltypes]`` as in
    test5.py:128-130.  emin/rmin2 as test5.py:132-133.  eplat/gplat are the
    plateau energies and d/d(dsq) gradients of test5.py:208-211; they are zero
    when ``shift_plateau`` is False, which is the "no potential grids" variant of
    the reference (test-nb-energrad.py:143-146).
    """
    rc = np.asarray(rc, np.float64)
    ac = np.asarray(ac, np.float64)
    ivor = np.asarray(ivor, np.float64)
    emin = -27.0 * ac ** 4 / (256.0 * rc ** 3)
    rmin2 = 4.0 * rc / (3.0 * ac)
    if rcap2 is None:
        rcap2 = np.zeros_like(rc)
    rcap2 = np.broadcast_to(np.asarray(rcap2, np.float64), rc.shape)
    p2 = float(plateau) ** 2
    if shift_plateau:
        eplat = nonbon(p2, rc, ac, emin, rmin2, ivor, rcap2)
        gplat = dnonbon_ddsq(p2, rc, ac, emin, rmin2, ivor, rcap2)
    else:
        eplat = np.zeros_like(rc)
        gplat = np.zeros_like(rc)
    t = np.stack([rc, ac, emin, rmin2, ivor, eplat, gplat, rcap2], axis=-1)  # [nr, nl, 8]
    return np.ascontiguousarray(np.transpose(t, (1, 0, 2)))  # [nl, nr, 8]


def _pp(pair, lt, rt):
    p = pair[lt, rt]
    return tuple(p[..., k] for k in range(8))


# --------------------------------------------------------------------------
# poses (test5.py:411-415; the Euler convention is pinned by the mono-leu data)
# --------------------------------------------------------------------------
def euler_to_Q(phi, psi, theta):
    """Column-convention rotation Q = Rz(phi) Ry(psi) Rz(-theta), [..., 3, 3]."""
    phi, psi, theta = np.broadcast_arrays(np.asarray(phi, np.float64),
                                          np.asarray(psi, np.float64),
                                          np.asarray(theta, np.float64))
    cp, sp = np.cos(phi), np.sin(phi)
    cs, ss = np.cos(psi), np.sin(psi)
    ct, st = np.cos(theta), np.sin(theta)
    Q = np.empty(phi.shape + (3, 3))
    Q[..., 0, 0] = cp * cs * ct + sp * st
    Q[..., 0, 1] = cp * cs * st - sp * ct
    Q[..., 0, 2] = cp * ss
    Q[..., 1, 0] = sp * cs * ct - cp * st
    Q[..., 1, 1] = sp * cs * st + cp * ct
    Q[..., 1, 2] = sp * ss
    Q[..., 2, 0] = -ss * ct
    Q[..., 2, 1] = -ss * st
    Q[..., 2, 2] = cs
    return Q


def euler_axes(phi, psi):
    """Rotation axes w_k with dQ/d(angle_k) = [w_k]x Q (k = phi, psi, theta)."""
    phi = np.asarray(phi, np.float64)
    psi = np.asarray(psi, np.float64)
    z = np.zeros_like(phi)
    w_phi = np.stack([z, z, z + 1.0], -1)
    w_psi = np.stack([-np.sin(phi), np.cos(phi), z], -1)
    w_theta = -np.stack([np.cos(phi) * np.sin(psi), np.sin(phi) * np.sin(psi), np.cos(psi)], -1)
    return np.stack([w_phi, w_psi, w_theta], -2)  # [..., 3, 3]


def pose_to_mat(pose):
    """(phi, psi, theta, t) -> the reference's row-vector 4x4 (test5.py:413-415)."""
    pose = np.asarray(pose, np.float64)
    mat = np.ones(pose.shape[:-1] + (4, 4))
    mat[..., :3, :3] = np.swapaxes(euler_to_Q(pose[..., 0], pose[..., 1], pose[..., 2]), -1, -2)
    mat[..., 3, :3] = pose[..., 3:6]
    return mat


def mat_to_euler(mat):
    """Inverse of ``pose_to_mat`` for proper rotations (used by fixtures/tests)."""
    mat = np.asarray(mat, np.float64)
    Q = np.swapaxes(mat[..., :3, :3], -1, -2)
    psi = np.arccos(np.clip(Q[..., 2, 2], -1.0, 1.0))
    phi = np.arctan2(Q[..., 1, 2], Q[..., 0, 2])
    theta = np.arctan2(-Q[..., 2, 1], -Q[..., 2, 0])
    return np.concatenate([np.stack([phi, psi, theta], -1), mat[..., 3, :3]], -1)


def transform(pose, lig):
    """Ligand beads moved by the pose, ``[x,1] @ mat`` (test5.py:315-317)."""
    pose = np.asarray(pose, np.float64)
    Q = euler_to_Q(pose[..., 0], pose[..., 1], pose[..., 2])
    return np.einsum("...ij,nj->...ni", Q, lig) + pose[..., None, 3:6]


# --------------------------------------------------------------------------
# potential grid term (test5.py:255-320)
# --------------------------------------------------------------------------
def _trilinear(grid_t, vox, quirk, dt):
    """8-corner trilinear interpolation of all 4 channels (test5.py:255-266).

    ``quirk=True`` uses the reference's floor/ceil weights: a coordinate that is
    an exact integer gets both weights 0 along that axis, so the bead reads 0.
    Returns (values [M,4], d(value ch0)/d(vox) [M,3]).
    """
    v0 = np.floor(vox)
    if quirk:
        v1 = np.ceil(vox)
        w0 = v1 - vox
        w1 = vox - v0
    else:
        v1 = v0 + 1.0
        w1 = vox - v0
        w0 = 1.0 - w1
    i0 = v0.astype(np.int64)
    i1 = v1.astype(np.int64)
    res = np.zeros((vox.shape[0], 4), dt)
    dres = np.zeros((vox.shape[0], 3), dt)
    # derivative of the weights along each axis (+1 for the upper corner)
    live = (w0 + w1) > 0  # per axis: False only at the quirk's integer points
    for cx in (0, 1):
        for cy in (0, 1):
            for cz in (0, 1):
                wx = w1[:, 0] if cx else w0[:, 0]
                wy = w1[:, 1] if cy else w0[:, 1]
                wz = w1[:, 2] if cz else w0[:, 2]
                ix = i1[:, 0] if cx else i0[:, 0]
                iy = i1[:, 1] if cy else i0[:, 1]
                iz = i1[:, 2] if cz else i0[:, 2]
                val = grid_t[np.arange(len(vox)), ix, iy, iz].astype(dt)
                w = (wx * wy * wz).astype(dt)
                res += w[:, None] * val
                sx = (1.0 if cx else -1.0) * live[:, 0]
                sy = (1.0 if cy else -1.0) * live[:, 1]
                sz = (1.0 if cz else -1.0) * live[:, 2]
                dres[:, 0] += sx * wy * wz * val[:, 0]
                dres[:, 1] += wx * sy * wz * val[:, 0]
                dres[:, 2] += wx * wy * sz * val[:, 0]
    return res, dres


class _TypeView:
    """Indexable view grid[type_of_row, x, y, z] without materialising copies."""

    def __init__(self, grid, types):
        self.grid, self.types, self.ndim = grid, types, 5

    def __getitem__(self, idx):
        rows, ix, iy, iz = idx
        return self.grid[self.types[rows], ix, iy, iz]


def grid_energrad(pos, gtype, geom, inner, outer, quirk=True, mode="reference", dtype=np.float64):
    """Per-bead grid energy and dE/dx (test5.py:286-311).

    pos [..., N, 3]; gtype [N] grid type slot per bead.  Inner grid if
    0 <= v < dim-1, else outer grid if 0 <= v_out < dim2-1, else 0
    (test5.py:288-294).  ``mode='reference'``: dE/dx = -interpolated stored
    force (test5.py:310).  ``mode='analytic'``: exact derivative of the
    interpolated energy channel.
    """
    dt = np.dtype(dtype)
    pos = np.asarray(pos, dt)
    shp = pos.shape[:-1]
    P = pos.reshape(-1, 3)
    types = np.broadcast_to(np.asarray(gtype), shp).reshape(-1)
    origin = np.asarray(geom["origin"], dt)
    spacing = dt.type(geom["spacing"])
    dim = np.asarray(geom["dim"])
    dim2 = np.asarray(geom["dim2"])
    v = (P - origin) / spacing
    inn = np.all((v >= 0) & (v < dim - 1), axis=1)
    vo = (v + dt.type(geom["extension"])) / dt.type(2)
    out = np.all((vo >= 0) & (vo < dim2 - 1), axis=1) & ~inn
    E = np.zeros(len(P), dt)
    G = np.zeros((len(P), 3), dt)
    for sel, vv, grid, scale in ((inn, v, inner, spacing), (out, vo, outer, spacing * 2)):
        if grid is None or not sel.any():
            continue
        idx = np.nonzero(sel)[0]
        res, dres = _trilinear(_TypeView(grid, types[idx]), vv[idx], quirk, dt)
        E[idx] = res[:, 0]
        if mode == "reference":
            G[idx] = -res[:, 1:4]
        else:
            G[idx] = dres / scale
    return E.reshape(shp), G.reshape(shp + (3,))


# --------------------------------------------------------------------------
# neighbour-grid pair term (test5.py:208-253, 322-349)
# --------------------------------------------------------------------------
def nb_energrad(pos, ltype, geom, nb_hdr, nb_list, rec, rtype, pair, mode="reference",
                dtype=np.float64, absolute=False):
    """Per-bead nbgrid pair energy and dE/dx.

    The list is looked up at the nearest inner-grid point ``floor(v+0.5)`` of a
    bead inside the inner grid (test5.py:322-336); each entry j != 65535 with
    d^2 < plateau^2 adds ``nonbon(d^2) - eplat`` (test5.py:213-215, 240) and
    the gradient of the custom JVP, ``2 d (dnonbon - gplat * p/|d|)``
    (test5.py:220-229).  ``mode='analytic'`` drops the plateau correction of
    the gradient (the exact derivative of the energy).  ``nb_hdr`` is
    ``[n_voxels, 2]`` (start, count) into ``nb_list``; ``geom["nb_refine"]`` = r
    > 1 puts the lists on the inner grid refined r times per axis (an
    extension: lists within plateau + the refined half-diagonal find the same
    pairs with fewer entries).  ``absolute=True`` sums the magnitudes of
    every additive component of each term instead of the term -- |rc/d^8| +
    |ac/d^6| + |emin term| + |plateau energy| for the energy, and likewise
    for the gradient -- the scale against which float32 rounding of the
    term is bounded (the components cancel near the potential's zero).
    """
    dt = np.dtype(dtype)
    pos = np.asarray(pos, dt)
    shp = pos.shape[:-1]
    P = pos.reshape(-1, 3)
    lt = np.broadcast_to(np.asarray(ltype), shp).reshape(-1)
    E = np.zeros(len(P), dt)
    G = np.zeros((len(P), 3), dt)
    if nb_hdr is None:
        return E.reshape(shp), G.reshape(shp + (3,))
    origin = np.asarray(geom["origin"], dt)
    spacing = dt.type(geom["spacing"])
    dim = np.asarray(geom["dim"])
    p = dt.type(geom["plateau"])
    v = (P - origin) / spacing
    inn = np.all((v >= 0) & (v < dim - 1), axis=1)
    idx = np.nonzero(inn)[0]
    if len(idx) == 0:
        return E.reshape(shp), G.reshape(shp + (3,))
    # nearest list-grid point: the inner grid point itself, or -- for lists
    # built on the inner grid refined r times per axis -- the refined point
    r = int(geom.get("nb_refine", 1))
    near = np.floor(v[idx] * r + dt.type(0.5)).astype(np.int64)
    ndim = (dim - 1) * r + 1
    vox = (near[:, 0] * ndim[1] + near[:, 1]) * ndim[2] + near[:, 2]
    start = nb_hdr[vox, 0].astype(np.int64)
    count = nb_hdr[vox, 1].astype(np.int64)
    tot = int(count.sum())
    if tot == 0:
        return E.reshape(shp), G.reshape(shp + (3,))
    bead = np.repeat(idx, count)
    first = np.repeat(np.cumsum(count) - count, count)
    ent = np.repeat(start, count) + (np.arange(tot) - first)
    j = nb_list[ent].astype(np.int64)
    ok = j != NB_EMPTY
    bead, j = bead[ok], j[ok]
    d = P[bead] - np.asarray(rec, dt)[j]
    dsq = (d * d).sum(1)
    m = dsq < p * p
    bead, j, d, dsq = bead[m], j[m], d[m], dsq[m]
    rc, ac, emin, rmin2, ivor, eplat, gplat, rcap2 = (x.astype(dt) for x in _pp(pair, lt[bead], rtype[j]))
    e = nonbon(dsq, rc, ac, emin, rmin2, ivor, rcap2) - eplat
    gmain = dnonbon_ddsq(dsq, rc, ac, emin, rmin2, ivor, rcap2)
    if mode == "reference":
        gfac = dt.type(2) * (gmain - gplat * p / np.sqrt(dsq))
    else:
        gfac = dt.type(2) * gmain
    gv = gfac[:, None] * d
    if absolute:
        dc = np.maximum(dsq, rcap2)
        rr2 = 1.0 / dc
        rr6 = rr2 ** 3
        near = dc < rmin2
        wiv = np.where(near, 1.0, np.abs(ivor))
        e = wiv * (np.abs(rc) * rr6 * rr2 + np.abs(ac) * rr6) + np.where(near, np.abs((ivor - 1.0) * emin), 0.0) \
            + np.abs(eplat)
        gm = np.where(dsq < rcap2, 0.0, wiv * rr2 ** 4 * (3.0 * np.abs(ac) + 4.0 * np.abs(rc) * rr2))
        if mode == "reference":
            gm = gm + np.abs(gplat) * p / np.sqrt(dsq)
        gv = 2.0 * gm[:, None] * np.abs(d)
    np.add.at(E, bead, e)
    np.add.at(G, bead, gv)
    return E.reshape(shp), G.reshape(shp + (3,))


# --------------------------------------------------------------------------
# pose energy / gradient (test5.py:404-429)
# --------------------------------------------------------------------------
def bead_energrad(X, lig_gtype, lig_ltype, G, mode="reference", quirk=True, dtype=np.float64):
    """Grid + nbgrid per-bead energies and dE/dx for transformed beads X [B,N,3]."""
    Eg, gg = grid_energrad(X, lig_gtype, G["geom"], G.get("inner"), G.get("outer"), quirk, mode, dtype)
    En, gn = nb_energrad(X, lig_ltype, G["geom"], G.get("nb_hdr"), G.get("nb_list"), G["rec"],
                         G["rtype"], G["pair"], mode, dtype)
    return Eg + En, gg + gn


def energrad(pose, lig, lig_gtype, lig_ltype, G, mode="reference", quirk=True, gravity=0.0,
             dtype=np.float64):
    """Per-pose energy and d E / d(phi, psi, theta, tx, ty, tz).

    E = E_grid + E_nb (+ gravity*|t|^2, test5.py:417-420); the pose gradient is
    the chain rule of test5.py:429's value_and_grad written out:
    dE/dt = sum_b dE/dx_b, dE/d(angle_k) = w_k . sum_b (x_b - t) x dE/dx_b.
    """
    pose = np.atleast_2d(np.asarray(pose, np.float64))
    X = transform(pose, np.asarray(lig, np.float64))
    Eb, gb = bead_energrad(X, lig_gtype, lig_ltype, G, mode, quirk, dtype)
    Eb = Eb.astype(np.float64)
    gb = gb.astype(np.float64)
    t = pose[:, 3:6]
    E = Eb.sum(1) + gravity * (t * t).sum(1)
    gt = gb.sum(1) + 2.0 * gravity * t
    tau = np.cross(X - t[:, None, :], gb).sum(1)
    W = euler_axes(pose[:, 0], pose[:, 1])
    ga = np.einsum("bkj,bj->bk", W, tau)
    return E, np.concatenate([ga, gt], 1)


def energrad_mat(mat, lig, lig_gtype, lig_ltype, G, mode="reference", quirk=True, dtype=np.float64):
    """Energy and dE/dmat for the reference's 4x4 row-vector poses (test1.py:409-412).

    dE/dmat[i, j] = sum_b [x_b, 1]_i dE/dx_b,j for j < 3; column 3 is unused.
    """
    mat = np.asarray(mat, np.float64).reshape(-1, 4, 4)
    lig = np.asarray(lig, np.float64)
    X = np.einsum("nk,bkl->bnl", np.concatenate([lig, np.ones((len(lig), 1))], 1), mat)[..., :3]
    Eb, gb = bead_energrad(X, lig_gtype, lig_ltype, G, mode, quirk, dtype)
    gb = gb.astype(np.float64)
    dmat = np.zeros_like(mat)
    dmat[:, :3, :3] = np.einsum("ni,bnj->bij", lig, gb)
    dmat[:, 3, :3] = gb.sum(1)
    return Eb.astype(np.float64).sum(1), dmat


# --------------------------------------------------------------------------
# quaternion call surface (test5.py:411-429) and the adabelief SCHEMA
# protocol (test5.py:14-23, 436-467)
# --------------------------------------------------------------------------
def _cross_matrix(v):
    z = np.zeros(v.shape[:-1])
    x, y, w = v[..., 0], v[..., 1], v[..., 2]
    return np.stack([np.stack([z, -w, y], -1), np.stack([w, z, -x], -1), np.stack([-y, x, z], -1)], -2)


def quat_to_matrix(q):
    """``Rotation.as_matrix()`` of scalar-last quaternions (the form JAX
    differentiates): R = (w^2 - v.v) I + 2 v v^T + 2 w [v]x."""
    q = np.asarray(q, np.float64)
    v, w = q[..., :3], q[..., 3]
    return ((w * w - (v * v).sum(-1))[..., None, None] * np.eye(3) + 2.0 * v[..., :, None] * v[..., None, :]
            + 2.0 * w[..., None, None] * _cross_matrix(v))


def quat_grad(q, dEdR):
    """dE/dq = sum_ij dE/dR_ij dR_ij/dq for :func:`quat_to_matrix`:
    dR/dw = 2 w I + 2 [v]x;  dR/dv_i = -2 v_i I + 2 (e_i v^T + v e_i^T) + 2 w [e_i]x."""
    q = np.asarray(q, np.float64)
    G = np.asarray(dEdR, np.float64)
    v, w = q[..., :3], q[..., 3]
    E = np.eye(3)
    out = np.zeros(q.shape)
    for i in range(3):
        ei = np.broadcast_to(E[i], v.shape)
        dR = (-2.0 * v[..., i][..., None, None] * E + 2.0 * (ei[..., :, None] * v[..., None, :]
              + v[..., :, None] * ei[..., None, :]) + 2.0 * w[..., None, None] * _cross_matrix(ei))
        out[..., i] = (G * dR).sum((-2, -1))
    dRw = 2.0 * w[..., None, None] * E + 2.0 * _cross_matrix(v)
    out[..., 3] = (G * dRw).sum((-2, -1))
    return out


def energrad_quat(q, t, lig_confs, conformers, lig_gtype, lig_ltype, G, gravity=0.0, mode="reference",
                  quirk=True, dtype=np.float64):
    """The reference's ``value_and_grad(main)`` (test5.py:411-429) for
    quaternion rotations: (E [B], dE/dq [B,4], dE/dt [B,3]).  The quaternion
    is normalised first (``Rotation.from_quat``); ``conformers`` index
    ``lig_confs [C,N,3]`` (test5.py:316); gravity*|t|^2 as test5.py:419."""
    q = np.asarray(q, np.float64)
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    t = np.asarray(t, np.float64)
    conformers = np.asarray(conformers, np.int64)
    mat = np.ones((len(q), 4, 4))
    mat[:, :3, :3] = quat_to_matrix(q)
    mat[:, 3, :3] = t
    E = np.zeros(len(q))
    dmat = np.zeros((len(q), 4, 4))
    for c in np.unique(conformers):
        sel = conformers == c
        E[sel], dmat[sel] = energrad_mat(mat[sel], lig_confs[c], lig_gtype, lig_ltype, G, mode, quirk, dtype)
    E = E + gravity * (t * t).sum(1)
    gt = dmat[:, 3, :3] + 2.0 * gravity * t
    return E, quat_grad(q, dmat[:, :3, :3]), gt


def minimise_schema(q, t, lig_confs, conformers, lig_gtype, lig_ltype, G, schema, gravity_weight=0.1,
                    b1=0.9, b2=0.999, eps=1e-16, eps_root=1e-16, dtype=np.float64):
    """test5.py:445-463: per stage (epochs, lr, gravity) a fresh
    optax.adabelief(lr) over (quaternion, translation).  optax's
    scale_by_belief: m <- b1 m + (1-b1) g;  s <- b2 s + (1-b2) (g - m_prev)^2
    + eps_root;  update = -lr (m / (1-b1^k)) / (sqrt(s / (1-b2^k)) + eps).
    After each update the quaternion is renormalised
    (``Rotation.from_quat(rotations.as_quat())``).  Returns (q, t, E) with E
    from the last evaluation, as the reference reports it (test5.py:465)."""
    q = np.array(q, np.float64)
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    t = np.array(t, np.float64)
    E = None
    for epochs, lr, grav in schema:
        mu = [np.zeros_like(q), np.zeros_like(t)]
        nu = [np.zeros_like(q), np.zeros_like(t)]
        for k in range(1, int(epochs) + 1):
            E, gq, gt = energrad_quat(q, t, lig_confs, conformers, lig_gtype, lig_ltype, G,
                                      gravity_weight if grav else 0.0, dtype=dtype)
            upd = []
            for i, g in enumerate((gq, gt)):
                err = g - mu[i]
                mu[i] = b1 * mu[i] + (1 - b1) * g
                nu[i] = b2 * nu[i] + (1 - b2) * err * err + eps_root
                upd.append(-lr * (mu[i] / (1 - b1 ** k)) / (np.sqrt(nu[i] / (1 - b2 ** k)) + eps))
            q = q + upd[0]
            t = t + upd[1]
            q = q / np.linalg.norm(q, axis=1, keepdims=True)
    return q, t, E


def allpairs_energrad(pose, lig, lig_ltype, rec, rtype, pair, rcut2=None, bead_grad=False):
    """Explicit all-pairs energy with its pose gradient: test-energy.py:46-58's
    sum of nonbon over every (ligand, receptor) pair within ``rcut2``, and the
    chain rule of :func:`energrad` (dE/dt = sum_b g_b, dE/d(angle_k) = w_k .
    sum_b (x_b - t) x g_b, g_b = sum_j 2 dnonbon/d(d^2) d_bj).  Also returns
    the per-pose sums of |energy term| and |gradient term| (1 + |x_b - t|),
    the float32 error scales of the parity tests.  Returns (E, grad, e_abs, g_abs),
    plus the per-bead dE/dx [B,N,3] with ``bead_grad``."""
    pose = np.atleast_2d(np.asarray(pose, np.float64))
    X = transform(pose, np.asarray(lig, np.float64))
    rec = np.asarray(rec, np.float64)
    prm = _pp(pair, np.asarray(lig_ltype)[:, None], np.asarray(rtype)[None, :])
    rc, ac, emin, rmin2, ivor, eplat, _, rcap2 = (np.asarray(v, np.float64) for v in prm)
    t = pose[:, 3:6]
    E = np.zeros(len(pose))
    ea = np.zeros(len(pose))
    ga = np.zeros(len(pose))
    gb = np.zeros_like(X)
    for b in range(len(pose)):
        d = X[b][:, None, :] - rec[None]
        dsq = (d * d).sum(-1)
        keep = np.ones_like(dsq, bool) if rcut2 is None else dsq < rcut2
        e = np.where(keep, nonbon(dsq, rc, ac, emin, rmin2, ivor, rcap2) - eplat, 0.0)
        g = np.where(keep, dnonbon_ddsq(dsq, rc, ac, emin, rmin2, ivor, rcap2), 0.0)
        E[b] = e.sum()
        ea[b] = np.abs(e).sum()
        gvec = 2.0 * g[..., None] * d
        gb[b] = gvec.sum(1)
        arm = 1.0 + np.linalg.norm(X[b] - t[b], axis=1)
        ga[b] = (np.abs(gvec).sum((1, 2)) * arm).sum()
    tau = np.cross(X - t[:, None, :], gb).sum(1)
    W = euler_axes(pose[:, 0], pose[:, 1])
    grad = np.concatenate([np.einsum("bkj,bj->bk", W, tau), gb.sum(1)], 1)
    return (E, grad, ea, ga, gb) if bead_grad else (E, grad, ea, ga)


def allpairs_energy(pose, lig, lig_ltype, rec, rtype, pair, rcut2=None):
    """Explicit all-pairs ATTRACT energy (test-energy.py:46-58; ATTRACT --rcut)."""
    X = transform(np.atleast_2d(pose), np.asarray(lig, np.float64))
    E = np.zeros(X.shape[0])
    for b in range(X.shape[0]):
        d = X[b][:, None, :] - np.asarray(rec, np.float64)[None]
        dsq = (d * d).sum(-1)
        rc, ac, emin, rmin2, ivor, _, _, rcap2 = _pp(pair, np.asarray(lig_ltype)[:, None], np.asarray(rtype)[None, :])
        e = nonbon(dsq, rc, ac, emin, rmin2, ivor, rcap2)
        if rcut2 is not None:
            e = np.where(dsq < rcut2, e, 0.0)
        E[b] = e.sum()
    return E


# --------------------------------------------------------------------------
# rigid-body ADAM minimiser (test4.py:440-455 with optax.adam; Euler DOF)
# --------------------------------------------------------------------------
def minimise(pose0, lig, lig_gtype, lig_ltype, G, steps, lr_rot=0.01, lr_trans=0.05, b1=0.9,
             b2=0.999, eps=1e-8, gravity=0.0, mode="reference", quirk=True, dtype=np.float64):
    """ADAM (Kingma & Ba; optax.adam's bias-corrected form, eps outside the sqrt).

    Each of ``steps`` iterations evaluates E and dE/dpose at the current pose and
    applies one update; a final evaluation gives the energy of the returned pose.
    Translation and rotation have their own learning rates.  A step whose
    gradient is not finite is skipped for that pose and flagged.
    Returns (pose, E_final, flags).
    """
    x = np.array(pose0, np.float64, copy=True).reshape(-1, 6)
    m = np.zeros_like(x)
    v = np.zeros_like(x)
    lr = np.array([lr_rot] * 3 + [lr_trans] * 3)
    flags = np.zeros(len(x), np.int32)
    for t in range(1, steps + 1):
        _, g = energrad(x, lig, lig_gtype, lig_ltype, G, mode, quirk, gravity, dtype)
        bad = ~np.all(np.isfinite(g), 1)
        flags |= bad.astype(np.int32)
        g = np.where(bad[:, None], 0.0, g)
        m1 = b1 * m + (1 - b1) * g
        v1 = b2 * v + (1 - b2) * g * g
        mh = m1 / (1 - b1 ** t)
        vh = v1 / (1 - b2 ** t)
        upd = lr * mh / (np.sqrt(vh) + eps)
        keep = bad[:, None]
        x = np.where(keep, x, x - upd)
        m = np.where(keep, m, m1)
        v = np.where(keep, v, v1)
    E, _ = energrad(x, lig, lig_gtype, lig_ltype, G, mode, quirk, gravity, dtype)
    return x, E, flags


# --------------------------------------------------------------------------
# grid builders (test-calc-grid-energy.py:90-196), small grids only
# --------------------------------------------------------------------------
def grid_points(geom, outer=False):
    """Cartesian positions of inner (origin + i*s) or outer ((2j - ext)*s + origin)
    grid points (test-calc-grid-energy.py:156-162), shape [dx, dy, dz, 3]."""
    o = np.asarray(geom["origin"], np.float64)
    s = float(geom["spacing"])
    if not outer:
        d = geom["dim"]
        ax = [o[k] + np.arange(d[k]) * s for k in range(3)]
    else:
        d = geom["dim2"]
        ax = [o[k] + (2.0 * np.arange(d[k]) - geom["extension"]) * s for k in range(3)]
    return np.stack(np.meshgrid(*ax, indexing="ij"), -1)


def build_potential_grid(rec, rtype, pair_full, geom, n_types, cutoff, outer=False, point_range=None):
    """Energy + force voxels ``[n_types, dx, dy, dz, 4]`` for ligand types 0..n_types-1.

    Per receptor bead within ``cutoff``: beyond the plateau, E(d) and force
    -2 dnonbon d; inside it, the plateau energy and the plateau force along d
    (what the nbgrid term's plateau correction removes again, test5.py:220-229).
    ``pair_full`` must carry the plateau values (eplat, gplat) for ``geom``.
    With ``point_range=(lo, hi)`` only those flat grid points are computed and
    ``[n_types, hi-lo, 4]`` is returned (for building a large grid in chunks).
    """
    pts = grid_points(geom, outer).reshape(-1, 3)
    lo, hi = (0, len(pts)) if point_range is None else point_range
    pts = pts[lo:hi]
    rec = np.asarray(rec, np.float64)
    p = float(geom["plateau"])
    out = np.zeros((n_types, len(pts), 4))
    from scipy.spatial import cKDTree

    tree = cKDTree(rec)
    lists = tree.query_ball_point(pts, cutoff)
    cnt = np.array([len(x) for x in lists])
    gi = np.repeat(np.arange(len(pts)), cnt)
    rj = np.concatenate([np.asarray(x, np.int64) for x in lists]) if cnt.sum() else np.zeros(0, np.int64)
    d = pts[gi] - rec[rj]
    dsq = (d * d).sum(1)
    inside = dsq < p * p
    dist = np.sqrt(dsq)
    for lt in range(n_types):
        rc, ac, emin, rmin2, ivor, eplat, gplat, rcap2 = _pp(pair_full, lt, np.asarray(rtype)[rj])
        e_far = nonbon(np.where(inside, p * p, dsq), rc, ac, emin, rmin2, ivor, rcap2)
        g_far = dnonbon_ddsq(np.where(inside, p * p, dsq), rc, ac, emin, rmin2, ivor, rcap2)
        e = np.where(inside, eplat, e_far)
        with np.errstate(divide="ignore", invalid="ignore"):
            scale = np.where(inside, np.where(dist > 0, gplat * p / dist, 0.0), g_far)
        f = -2.0 * scale[:, None] * d
        out[lt, :, 0] = np.bincount(gi, e, minlength=len(pts))
        for k in range(3):
            out[lt, :, 1 + k] = np.bincount(gi, f[:, k], minlength=len(pts))
    if point_range is not None:
        return out
    d3 = geom["dim2"] if outer else geom["dim"]
    return out.reshape((n_types,) + tuple(int(x) for x in d3) + (4,))


def build_nbgrid(rec, geom, radius):
    """Neighbour lists at inner grid points (CSR): receptor beads within
    ``radius`` of origin + i*s, ascending index.  Returns (hdr [V,2] u32, list u16)."""
    from scipy.spatial import cKDTree

    pts = grid_points(geom, False).reshape(-1, 3)
    tree = cKDTree(np.asarray(rec, np.float64))
    lists = tree.query_ball_point(pts, radius)
    cnt = np.array([len(x) for x in lists], np.int64)
    start = np.cumsum(cnt) - cnt
    flat = np.concatenate([np.sort(np.asarray(x, np.int64)) for x in lists]) if cnt.sum() else np.zeros(0, np.int64)
    hdr = np.stack([start, cnt], 1).astype(np.uint32)
    return hdr, flat.astype(np.uint16)


def build_nbgrid_f32(rec32, origin32, spacing32, dim, radius32):
    """Neighbour lists with the builder kernel's float32 arithmetic, bit for bit.

    The same membership rule as :func:`build_nbgrid` (receptor beads within
    ``radius`` of grid point origin + i*s, test-calc-grid-energy.py:90-103),
    computed as the GPU builder computes it: the point as
    ``fl(origin + fl(i * s))``, the squared distance as
    ``fl(fl(fl(dx*dx) + fl(dy*dy)) + fl(dz*dz))`` with ``dx = fl(x - r_x)``, and
    the test ``d2 <= fl(radius * radius)``, every operation rounded to float32
    on its own.  ``rec32`` [R, 3] float32 in the order the lists index; the
    entries of a point are in ascending index order.  A float64 KD-tree query
    with a margin picks the candidates; the float32 test decides.
    """
    from scipy.spatial import cKDTree

    f = np.float32
    rec32 = np.asarray(rec32, f).reshape(-1, 3)
    o = np.asarray(origin32, f).reshape(3)
    s = f(spacing32)
    r2 = f(radius32) * f(radius32)
    dim = [int(d) for d in dim]
    ax = [o[k] + np.arange(dim[k], dtype=f) * s for k in range(3)]  # each a rounded product, then sum
    pts = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 3)
    tree = cKDTree(rec32.astype(np.float64))
    cand = tree.query_ball_point(pts.astype(np.float64), float(np.sqrt(np.float64(r2))) + 1e-3)
    cnt = np.array([len(x) for x in cand], np.int64)
    gi = np.repeat(np.arange(len(pts)), cnt)
    rj = np.concatenate([np.asarray(x, np.int64) for x in cand]) if cnt.sum() else np.zeros(0, np.int64)
    d = pts[gi] - rec32[rj]  # float32, rounded per component
    dsq = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    keep = dsq <= r2
    gi, rj = gi[keep], rj[keep]
    order = np.lexsort((rj, gi))
    gi, rj = gi[order], rj[order]
    n = np.bincount(gi, minlength=len(pts)).astype(np.int64)
    start = np.cumsum(n) - n
    hdr = np.stack([start, n], 1).astype(np.uint32)
    return hdr, rj.astype(np.uint16)


def repack_bricks(inner, outer):
    """Brick layout: for each type, every inner then every outer base voxel
    (x,y,z) with x<dim-1.. holds its 8 corners (cx,cy,cz) in order cx*4+cy*2+cz.
    Returns float32 [n_types, n_inner_bricks + n_outer_bricks, 8, 4]."""
    parts = []
    for g in (inner, outer):
        if g is None:
            continue
        T, dx, dy, dz, _ = g.shape
        b = np.empty((T, dx - 1, dy - 1, dz - 1, 8, 4), np.float32)
        for c in range(8):
            cx, cy, cz = (c >> 2) & 1, (c >> 1) & 1, c & 1
            b[:, :, :, :, c] = g[:, cx:cx + dx - 1, cy:cy + dy - 1, cz:cz + dz - 1]
        parts.append(b.reshape(T, -1, 8, 4))
    return np.concatenate(parts, 1)
