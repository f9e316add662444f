"""Receptor grids resident in HBM.

A :class:`Grid` holds, on one CUDA device:

* ``bricks``  -- the potential grids (inner + outer, every ligand type) repacked
  so that the 8 trilinear corners of a voxel are one contiguous, 128-byte
  aligned run of float4 ``(E, Fx, Fy, Fz)``: one 128-B bulk copy per bead,
  made only when the bead enters another cell;
* ``nb_hdr`` / ``nb_list`` -- the neighbour grid as CSR: ``{start, count}`` per
  list-grid point (the inner grid, or the inner grid refined ``nb_refine``
  times) and uint16 receptor indices (65535 = empty slot), with the fixed-size
  records ``nb_rec`` the kernels copy;
* ``rec`` -- receptor beads ``x, y, z, type`` (float4, type as int32 bits);
* ``pair`` -- the per-pair parameter table for this grid's plateau.

The dense layout of the reference (read_grid2.py:92-155:
``inner_potential_grid [T, dx, dy, dz, 4]``, ``outer_potential_grid``,
``nr_neighbours``/``neighbour_grid``) is accepted by :meth:`Grid.from_dense`;
:meth:`Grid.build` computes everything from receptor beads on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .forcefield import ForceField


@dataclass
class GridGeom:
    origin: tuple
    spacing: float
    dim: tuple
    dim2: tuple
    extension: int
    plateau: float
    n_types: int

    def to_c(self) -> _lib.AttGridGeom:
        g = _lib.AttGridGeom()
        for k in range(3):
            g.origin[k] = float(self.origin[k])
            g.dim[k] = int(self.dim[k])
            g.dim2[k] = int(self.dim2[k])
        g.spacing = float(self.spacing)
        g.extension = int(self.extension)
        g.plateau = float(self.plateau)
        g.n_types = int(self.n_types)
        return g

    @property
    def n_voxels(self) -> int:
        return int(np.prod(self.dim))

    def refined(self, r: int) -> "GridGeom":
        """The inner grid refined r times per axis (the neighbour-list grid of
        ``nb_refine = r``): same origin, spacing / r, (dim - 1) * r + 1 points."""
        if r <= 1:
            return self
        return GridGeom(self.origin, self.spacing / r, tuple((int(d) - 1) * r + 1 for d in self.dim), (0, 0, 0),
                        self.extension, self.plateau, self.n_types)

    @property
    def n_inner_bricks(self) -> int:
        return int(np.prod(np.asarray(self.dim) - 1))

    @property
    def n_outer_bricks(self) -> int:
        d = np.asarray(self.dim2)
        return int(np.prod(d - 1)) if np.all(d >= 2) else 0

    def as_dict(self) -> dict:
        return dict(origin=np.asarray(self.origin, np.float64), spacing=float(self.spacing),
                    dim=np.asarray(self.dim), dim2=np.asarray(self.dim2), extension=int(self.extension),
                    plateau=float(self.plateau))

    @classmethod
    def around(cls, centre, radius, spacing=0.9, padding=10.0, extension=32, plateau=5.0, n_types=32):
        """Cubic inner grid covering a sphere plus padding; the outer grid (twice
        the spacing) reaches ``extension`` inner spacings further on every side."""
        half = radius + padding
        n = int(np.ceil(2 * half / spacing)) + 1
        origin = np.asarray(centre, np.float64) - (n - 1) * spacing / 2.0
        n2 = int(np.ceil((n - 1 + 2 * extension) / 2.0)) + 1
        return cls(tuple(origin), spacing, (n, n, n), (n2, n2, n2), extension, plateau, n_types)


def _dev(device):
    """A torch.device with its index resolved (``cuda`` -> ``cuda:<current>``)."""
    d = torch.device(device if device is not None else "cuda")
    if d.type == "cuda" and d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    return d


def pack_receptor(xyz, rtype, device) -> torch.Tensor:
    xyz = np.asarray(xyz, np.float32).reshape(-1, 3)
    rtype = np.asarray(rtype, np.int32).reshape(-1)
    if len(xyz) != len(rtype):
        raise ValueError("receptor coordinates and types differ in length")
    if len(xyz) >= _lib.ATT_NB_EMPTY:
        raise ValueError(f"{len(xyz)} receptor beads: at most 65534 fit the uint16 neighbour lists")
    a = np.zeros((max(len(xyz), 1), 4), np.float32)
    a[: len(xyz), :3] = xyz
    a[: len(xyz), 3] = rtype.view(np.float32)
    return torch.from_numpy(a).to(device)


def spatial_order(xyz, bits: int = 10) -> np.ndarray:
    """Permutation putting points in Morton (Z-curve) order of their position
    quantised to 2**bits cells per axis of the bounding box."""
    x = np.asarray(xyz, np.float64).reshape(-1, 3)
    if len(x) == 0:
        return np.zeros(0, np.int64)
    lo = x.min(0)
    span = max(float(np.ptp(x, 0).max()), 1e-9)
    q = np.minimum(((x - lo) / span * ((1 << bits) - 1) + 0.5).astype(np.int64), (1 << bits) - 1)
    code = np.zeros(len(x), np.int64)
    for b in range(bits):
        for k in range(3):
            code |= ((q[:, k] >> b) & 1) << (3 * b + k)
    return np.argsort(code, kind="stable")


class Grid:
    """One receptor (potential grids + neighbour grid + beads) on the device.

    The receptor beads are held on the device in Morton order of their
    positions (``rec_perm``: device position -> given index), and the
    neighbour lists name beads by device position: the beads one warp's
    lists name then share few cache lines.  ``rec_xyz``/``rec_type`` and
    :meth:`dense_host` keep the caller's order.
    """

    def __init__(self, geom: GridGeom, rec_xyz, rec_type, ff: ForceField, *, bricks=None, nb_hdr=None,
                 nb_list=None, inner=None, outer=None, shift_plateau=None, device=None, list_space="given",
                 nb_refine: int = 1):
        self.device = _dev(device)
        self.geom = geom
        self.ff = ff
        if nb_refine not in (1, 2, 4):
            raise ValueError("nb_refine must be 1, 2 or 4")
        self.nb_refine = nb_refine
        self.nb_geom = geom.refined(nb_refine)  # the grid the neighbour lists sit on
        rec_type = np.asarray(rec_type, np.int64)
        if len(rec_type) and (rec_type.min() < 0 or rec_type.max() >= ff.n_rtypes):
            raise ValueError("receptor type outside the force field")
        self.n_rec = len(rec_type)
        self.rec_xyz = np.asarray(rec_xyz, np.float64).reshape(-1, 3)
        self.rec_type = rec_type
        self.rec_perm = spatial_order(self.rec_xyz)
        self.rec = pack_receptor(self.rec_xyz[self.rec_perm], rec_type[self.rec_perm], self.device)
        if nb_list is not None and list_space == "given" and self.n_rec:
            lut = torch.full((1 << 16,), _lib.ATT_NB_EMPTY, dtype=torch.int32, device=self.device)
            inv = np.empty(self.n_rec, np.int64)
            inv[self.rec_perm] = np.arange(self.n_rec)
            lut[: self.n_rec] = torch.from_numpy(inv.astype(np.int32)).to(self.device)
            nb_list = lut[nb_list.to(torch.int64) & 0xFFFF].to(torch.int16)
        self.bricks = bricks
        self.inner = inner
        self.outer = outer
        self.nb_hdr = nb_hdr
        self.nb_list = nb_list
        if shift_plateau is None:
            shift_plateau = bricks is not None
        self.shift_plateau = shift_plateau
        self.pair = torch.from_numpy(ff.pair_table(geom.plateau, shift_plateau)).to(self.device)
        # versions of the dense grids the bricks were packed from (autograd.py)
        self._packed_version = (None if inner is None else inner._version,
                                None if outer is None else outer._version)
        self.nb_rec = None
        self.nb_rec_bytes = 0
        if nb_hdr is not None:
            self._pack_records()
        self._att = None

    def _pack_records(self, rec_bytes: int | None = None):
        """Fixed-size neighbour records (copied with the brick per bead and step): the
        smallest of 32/64/128 bytes whose inline entries hold 99 % of the
        non-empty lists; longer lists continue in the CSR list."""
        counts = self.nb_hdr[:, 1]
        if rec_bytes is None:
            nz = counts[counts > 0].to(torch.float32)
            q = float(torch.quantile(nz[: 1 << 24], 0.99).item()) if nz.numel() else 0.0
            rec_bytes = next((b for b in (32, 64, 128) if (b - 6) // 2 >= q), 128)
        self.nb_rec_bytes = rec_bytes
        self.nb_rec = torch.empty(self.nb_geom.n_voxels * rec_bytes, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            st = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(_lib.load().att_nbgrid_pack_records(_lib.ptr(self.nb_hdr), _lib.ptr(self.nb_list),
                                                           self.nb_geom.n_voxels, rec_bytes, _lib.ptr(self.nb_rec),
                                                           st), "att_nbgrid_pack_records")

    # ------------------------------------------------------------------ C view
    def att(self) -> _lib.AttGrid:
        if self._att is None:
            a = _lib.AttGrid()
            a.geom = self.geom.to_c()
            a.bricks = _lib.ptr(self.bricks)
            a.n_inner_bricks = self.geom.n_inner_bricks
            a.n_outer_bricks = self.n_outer_bricks_used
            a.nb_hdr = _lib.ptr(self.nb_hdr)
            a.nb_list = _lib.ptr(self.nb_list)
            a.n_nb_entries = 0 if self.nb_list is None else self.nb_list.numel()
            a.rec = _lib.ptr(self.rec)
            a.n_rec = self.n_rec
            a.n_rtypes = self.ff.n_rtypes
            a.n_ltypes = self.ff.n_ltypes
            a.pair = _lib.ptr(self.pair)
            a.nb_rec = _lib.ptr(self.nb_rec)
            a.nb_rec_bytes = self.nb_rec_bytes
            a.nb_refine = self.nb_refine
            self._att = a
        return self._att

    @property
    def n_outer_bricks_used(self) -> int:
        if self.bricks is None:
            return 0
        return int(self.bricks.shape[1]) - self.geom.n_inner_bricks

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in (self.bricks, self.nb_hdr, self.nb_list, self.rec,
                                                            self.pair, self.inner, self.outer, self.nb_rec)
                   if t is not None)

    # ------------------------------------------------------------ constructors
    @classmethod
    def from_dense(cls, geom: GridGeom, rec_xyz, rec_type, ff: ForceField, inner=None, outer=None,
                   nb_hdr=None, nb_list=None, neighbour_grid=None, nr_neighbours=None, shift_plateau=None,
                   keep_dense=False, device=None, nb_refine: int = 1):
        """Grid from the reference's dense arrays (read_grid2.py:92-155).

        ``inner``/``outer``: float ``[T, dx, dy, dz, 4]`` (E, Fx, Fy, Fz), or None.
        The neighbour grid is CSR (``nb_hdr [V,2]``, ``nb_list``) or the dense padded
        ``neighbour_grid [dx,dy,dz,maxnb]`` uint16 with ``nr_neighbours`` (negative = 0),
        at the inner grid points (the reference's layout) or, with ``nb_refine``
        = 2 or 4, at the points of :meth:`GridGeom.refined`.
        """
        ngeom = geom.refined(nb_refine)
        dev = _dev(device)
        lib = _lib.load()
        bricks = inner_t = outer_t = None
        if inner is not None:
            inner_t = torch.as_tensor(np.ascontiguousarray(inner, np.float32)).to(dev)
            if tuple(inner_t.shape) != (geom.n_types, *geom.dim, 4):
                raise ValueError(f"inner grid shape {tuple(inner_t.shape)} != {(geom.n_types, *geom.dim, 4)}")
            if outer is not None:
                outer_t = torch.as_tensor(np.ascontiguousarray(outer, np.float32)).to(dev)
                if tuple(outer_t.shape) != (geom.n_types, *geom.dim2, 4):
                    raise ValueError("outer grid shape does not match dim2")
            bricks = _alloc_bricks(geom, outer_t is not None, dev)
            gc = geom.to_c()
            with torch.cuda.device(dev):
                st = torch.cuda.current_stream(dev).cuda_stream
                _lib.check(lib.att_grid_repack(C.byref(gc), _lib.ptr(inner_t), _lib.ptr(outer_t),
                                               _lib.ptr(bricks), st), "att_grid_repack")
        hdr_t = lst_t = None
        if neighbour_grid is not None:
            ng = np.asarray(neighbour_grid).reshape(ngeom.n_voxels, -1)
            nr = np.maximum(np.asarray(nr_neighbours, np.int64).reshape(-1), 0)
            nr = np.minimum(nr, ng.shape[1])
            start = np.cumsum(nr) - nr
            mask = np.arange(ng.shape[1])[None, :] < nr[:, None]
            nb_list = ng[mask].astype(np.uint16)
            nb_hdr = np.stack([start, nr], 1)
        if nb_hdr is not None:
            nb_hdr = np.asarray(nb_hdr, np.int64)
            nb_list = np.asarray(nb_list, np.uint16)
            if nb_hdr.shape != (ngeom.n_voxels, 2):
                raise ValueError("nb_hdr must be [list-grid points, 2]")
            if len(nb_hdr) and (nb_hdr[:, 0] + nb_hdr[:, 1]).max() > len(nb_list):
                raise ValueError("neighbour list header points past the list")
            hdr_t = torch.from_numpy(nb_hdr.astype(np.uint32).view(np.int32)).to(dev)
            lst = nb_list if len(nb_list) else np.full(1, _lib.ATT_NB_EMPTY, np.uint16)
            lst_t = torch.from_numpy(lst.view(np.int16)).to(dev)
        g = cls(geom, rec_xyz, rec_type, ff, bricks=bricks, nb_hdr=hdr_t, nb_list=lst_t,
                inner=inner_t if keep_dense else None, outer=outer_t if keep_dense else None,
                shift_plateau=shift_plateau, device=dev, nb_refine=nb_refine)
        return g

    @classmethod
    def build(cls, rec_xyz, rec_type, ff: ForceField, geom: GridGeom, cutoff: float = 10.0,
              list_radius: float | None = None, outer: bool = True, potentials: bool = True,
              keep_dense: bool = False, device=None, nb_refine: int = 4):
        """Build potential grids (K3), neighbour lists (K4) and bricks (K5) on the GPU.

        The neighbour lists sit on the inner grid refined ``nb_refine`` times per
        axis and hold every receptor bead within ``list_radius`` of a list-grid
        point (default: plateau + half the list grid's voxel diagonal, so that
        no pair closer than the plateau is missed by the nearest-point lookup).
        The pairs found do not depend on ``nb_refine``; a finer list grid visits
        fewer entries beyond the plateau (2: ~19 % fewer than 1, 4: another
        ~10 % fewer than 2) for 8x / 64x the record memory of the inner grid
        (a 2500-bead receptor in a 40 A sphere: 0.36 GB at 2, 2.9 GB at 4).
        """
        dev = _dev(device)
        lib = _lib.load()
        if potentials and geom.n_types > ff.n_ltypes:
            raise ValueError("grid has more potential slots than the force field has ligand types")
        if nb_refine not in (1, 2, 4):
            raise ValueError("nb_refine must be 1, 2 or 4")
        ngeom = geom.refined(nb_refine)
        if list_radius is None:
            list_radius = geom.plateau + ngeom.spacing * np.sqrt(3.0) / 2.0 + 1e-3
        perm = spatial_order(rec_xyz)  # the order Grid.__init__ puts the beads in
        rec = pack_receptor(np.asarray(rec_xyz, np.float64).reshape(-1, 3)[perm], np.asarray(rec_type)[perm], dev)
        n_rec = len(np.asarray(rec_type).reshape(-1))
        gc = geom.to_c()
        with torch.cuda.device(dev):
            st = torch.cuda.current_stream(dev).cuda_stream
            inner_t = outer_t = bricks = None
            if potentials:
                full = torch.from_numpy(ff.pair_table(geom.plateau, True)).to(dev)
                inner_t = torch.empty((geom.n_types, *geom.dim, 4), dtype=torch.float32, device=dev)
                _lib.check(lib.att_build_potential_grid(C.byref(gc), _lib.ptr(rec), n_rec, _lib.ptr(full),
                                                        ff.n_rtypes, geom.n_types, float(cutoff), 0,
                                                        _lib.ptr(inner_t), st), "build inner grid")
                if outer and min(geom.dim2) >= 2:
                    outer_t = torch.empty((geom.n_types, *geom.dim2, 4), dtype=torch.float32, device=dev)
                    _lib.check(lib.att_build_potential_grid(C.byref(gc), _lib.ptr(rec), n_rec, _lib.ptr(full),
                                                            ff.n_rtypes, geom.n_types, float(cutoff), 1,
                                                            _lib.ptr(outer_t), st), "build outer grid")
                bricks = _alloc_bricks(geom, outer_t is not None, dev)
                _lib.check(lib.att_grid_repack(C.byref(gc), _lib.ptr(inner_t), _lib.ptr(outer_t),
                                               _lib.ptr(bricks), st), "att_grid_repack")
            nvox = ngeom.n_voxels
            ngc = ngeom.to_c()
            hdr = torch.empty((nvox, 2), dtype=torch.int32, device=dev)
            total = torch.zeros(1, dtype=torch.int64, device=dev)
            wsb = lib.att_nbgrid_workspace_bytes(nvox)
            ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
            _lib.check(lib.att_nbgrid_count(C.byref(ngc), _lib.ptr(rec), n_rec, float(list_radius), _lib.ptr(hdr),
                                            _lib.ptr(total), _lib.ptr(ws), wsb, st), "att_nbgrid_count")
            n_ent = int(total.item())
            check_list_total(n_ent)
            lst = torch.empty(max(n_ent, 1), dtype=torch.int16, device=dev)
            _lib.check(lib.att_nbgrid_fill(C.byref(ngc), _lib.ptr(rec), n_rec, float(list_radius), _lib.ptr(hdr),
                                           _lib.ptr(lst), st), "att_nbgrid_fill")
        g = cls(geom, rec_xyz, rec_type, ff, bricks=bricks, nb_hdr=hdr, nb_list=lst,
                inner=inner_t if keep_dense else None, outer=outer_t if keep_dense else None,
                shift_plateau=potentials, device=dev, list_space="device", nb_refine=nb_refine)
        g.list_radius = list_radius
        g.cutoff = cutoff
        return g

    def nb_entries(self) -> int:
        return 0 if self.nb_list is None else self.nb_list.numel()

    def dense_host(self):
        """(inner, outer, nb_hdr, nb_list) as NumPy arrays (for checks), the
        lists naming beads by the caller's index, ascending per grid point."""
        f = lambda t: None if t is None else t.detach().cpu().numpy()
        hdr = None if self.nb_hdr is None else f(self.nb_hdr).view(np.uint32)
        lst = None if self.nb_list is None else f(self.nb_list).view(np.uint16).copy()
        if lst is not None and self.n_rec:
            total = int(hdr[:, 1].astype(np.int64).sum())
            body = lst[:total].astype(np.int64)
            ok = body < self.n_rec
            body[ok] = self.rec_perm[body[ok]]
            body[~ok] = _lib.ATT_NB_EMPTY
            vox = np.repeat(np.arange(len(hdr)), hdr[:, 1].astype(np.int64))
            start = hdr[:, 0].astype(np.int64)
            if np.array_equal(start, np.cumsum(hdr[:, 1].astype(np.int64)) - hdr[:, 1]):
                lst[:total] = body[np.lexsort((body, vox))]
            else:  # general CSR: sort each list in place
                for v in np.flatnonzero(hdr[:, 1]):
                    s0, n = int(start[v]), int(hdr[v, 1])
                    vals = lst[s0:s0 + n].astype(np.int64)
                    ok = vals < self.n_rec
                    vals[ok] = self.rec_perm[vals[ok]]
                    lst[s0:s0 + n] = np.sort(vals)
        return f(self.inner), f(self.outer), hdr, lst


def check_list_total(n_entries: int) -> None:
    """The neighbour lists' CSR starts are 32-bit (``AttGrid.nb_hdr``): a grid
    whose entry total exceeds 2**32 - 1 would wrap them, so it is refused."""
    if n_entries > 0xFFFFFFFF:
        raise ValueError(f"{n_entries} neighbour-list entries: the 32-bit list starts hold at most 2**32 - 1; "
                         "use a coarser list grid (nb_refine) or a smaller list radius")


def _alloc_bricks(geom: GridGeom, with_outer: bool, dev) -> torch.Tensor:
    nb = geom.n_inner_bricks + (geom.n_outer_bricks if with_outer else 0)
    # float32 [T][bricks][8][4]; torch's allocator returns 512-B aligned blocks
    t = torch.empty((geom.n_types, nb, 8, 4), dtype=torch.float32, device=dev)
    assert t.data_ptr() % 128 == 0
    return t
