"""ATTRACT binary docking grids (``.grid``): reader and writer.

``read_grid(grid_data, read_gradients)`` has the name, arguments and result of
the reference's ``read_grid2.read_grid`` (read_grid2.py:16-161): a namedtuple
``Grid`` with the fields ``gridspacing, gridextension, plateaudis,
neighbourdis, alphabet, origin, dim, dim2, natoms, inner_potential_grid,
nr_neighbours, max_nr_neighbours, neighbour_grid, outer_potential_grid,
neighbour_grid_ravel``, built with vectorised NumPy instead of per-slot loops.
``read_grid_csr`` returns the neighbour grid as the CSR pair that
:class:`attract_b200.Grid` consumes, without the padded dense array.
``write_grid`` produces the same format from dense arrays (round trip).

File layout (native little-endian, fields packed without padding, as
read_grid2.py:41-68 reads them one scalar at a time):

==========================  ==============================================
``?``  is_torquegrid        must be false
``h``  arch                 64
``d``  gridspacing, ``i`` gridextension, ``d`` plateaudis, ``d`` neighbourdis
``?`` x 99 alphabet         potential present per ATTRACT type 1..99
``f`` x 3 origin, ``i`` x 3 dim, ``i`` x 3 dim2, ``i`` natoms, ``d`` x 3 pivot
``i`` nr_energrads, ``i`` -1  then float32 [nr_energrads][4] (E, Fx, Fy, Fz)
``i`` nr_neighbours, ``i`` -1 then {u8 type, u32 index} (8 B, aligned) each
``q`` innergridsize         then per inner point (x fastest) {u32 potential[100],
                            i32 neighbourlist (1-based), i16 nr_neighbours} (408 B)
``q`` biggridsize           then per outer point (x fastest) u32 potential[100]
==========================  ==============================================

A potential index is 1-based into the energrads; 0 in the outer grid means
"no value" (reads as zeros).  Slot 99 (the electrostatic potential) is ignored.
"""
from __future__ import annotations

import struct
from collections import namedtuple

import numpy as np

_HEAD = struct.Struct("=?hdidd99?3f3i3ii3d")
_NB_DTYPE = np.dtype([("type", np.uint8), ("index", np.uint32)], align=True)
_INNER_DTYPE = np.dtype([("potential", np.uint32, 100), ("neighbourlist", np.int32), ("nr_neighbours", np.int16)],
                        align=True)

GRID_FIELDS = ("gridspacing", "gridextension", "plateaudis", "neighbourdis", "alphabet", "origin", "dim", "dim2",
               "natoms", "inner_potential_grid", "nr_neighbours", "max_nr_neighbours", "neighbour_grid",
               "outer_potential_grid", "neighbour_grid_ravel")
GridTuple = namedtuple("Grid", GRID_FIELDS)


class GridFileError(ValueError):
    """The bytes are not an ATTRACT grid this reader supports."""


def _parse(grid_data: bytes, read_gradients: bool):
    buf = memoryview(grid_data)
    if len(buf) < _HEAD.size:
        raise GridFileError("truncated grid header")
    h = _HEAD.unpack_from(buf, 0)
    torque, arch = h[0], h[1]
    if torque:
        raise GridFileError("torque grids are not supported")
    if arch != 64:
        raise GridFileError(f"grid written for a {arch}-bit architecture (64 expected)")
    d = {"gridspacing": h[2], "gridextension": h[3], "plateaudis": h[4], "neighbourdis": h[5],
         "alphabet": np.array(h[6:105], bool), "origin": np.array(h[105:108], np.float64),
         "dim": np.array(h[108:111]), "dim2": np.array(h[111:114]), "natoms": h[114]}
    pos = _HEAD.size
    if np.any(d["dim"] < 1) or np.any(d["dim2"] < 0):
        raise GridFileError(f"grid dimensions {list(d['dim'])} / {list(d['dim2'])} out of range")

    def ints(n):
        nonlocal pos
        if pos + 4 * n > len(buf):
            raise GridFileError("truncated grid")
        v = struct.unpack_from(f"={n}i", buf, pos)
        pos += 4 * n
        return v

    def array(dtype, count):
        nonlocal pos
        if count < 0 or pos + np.dtype(dtype).itemsize * count > len(buf):
            raise GridFileError("truncated grid")
        a = np.frombuffer(buf, dtype=dtype, count=count, offset=pos)
        pos += a.nbytes
        return a

    def long():
        nonlocal pos
        if pos + 8 > len(buf):
            raise GridFileError("truncated grid")
        (v,) = struct.unpack_from("=q", buf, pos)
        pos += 8
        return v

    n_eg, shm = ints(2)
    energrads = np.zeros((0, 4), np.float32)
    if n_eg:
        if shm != -1:
            raise GridFileError("grid refers to shared memory")
        energrads = array(np.float32, n_eg * 4).reshape(n_eg, 4)
    n_nb, shm = ints(2)
    if shm != -1:
        raise GridFileError("grid refers to shared memory")
    neighbours = array(_NB_DTYPE, n_nb)["index"]
    inner_size = long()
    dx, dy, dz = (int(v) for v in d["dim"])
    if inner_size != dx * dy * dz:
        raise GridFileError(f"inner grid size {inner_size} != {dx}*{dy}*{dz}")
    inner = array(_INNER_DTYPE, inner_size)
    if len(neighbours) and neighbours.max() >= 2 ** 16:
        raise GridFileError("too many atoms for uint16 neighbour lists")
    big_size = long()
    big = None
    if n_eg:
        dx2, dy2, dz2 = (int(v) for v in d["dim2"])
        if big_size != dx2 * dy2 * dz2:
            raise GridFileError(f"outer grid size {big_size} != {dx2}*{dy2}*{dz2}")
        big = array(np.uint32, big_size * 100).reshape(big_size, 100)
    elif big_size != 0:
        raise GridFileError("outer grid without energrads")

    present = np.flatnonzero(d["alphabet"][:99])
    chan = slice(None) if read_gradients else 0

    def potentials(idx, dims, outer):
        # idx: [points (x fastest), 100] -> [n_potentials, x, y, z(, 4)]
        if np.any(idx[:, np.flatnonzero(~d["alphabet"][:99])] != 0):
            raise GridFileError("potential index for a type outside the alphabet")
        sel = idx[:, present].T.astype(np.int64)  # [T, points]
        if np.any(sel > len(energrads)) or (not outer and np.any(sel < 1)):
            raise GridFileError("potential index outside the energrads")
        vals = np.where(sel[..., None] > 0, energrads[np.maximum(sel - 1, 0)], 0.0).astype(np.float32)
        a, b, c = dims
        vals = vals.reshape(len(present), c, b, a, 4).transpose(0, 3, 2, 1, 4)
        return np.ascontiguousarray(vals[..., chan])

    if n_eg:
        d["inner_potential_grid"] = potentials(inner["potential"], (dx, dy, dz), False)
    # neighbour lists: per inner point (x fastest in the file) a 1-based start and a count
    nr = inner["nr_neighbours"].astype(np.int64)
    start = inner["neighbourlist"].astype(np.int64) - 1
    to_xyz = lambda a: np.ascontiguousarray(a.reshape(dz, dy, dx).transpose(2, 1, 0))
    d["nr_neighbours"] = to_xyz(inner["nr_neighbours"])
    cnt = to_xyz(np.maximum(nr, 0)).reshape(-1)
    st = to_xyz(start).reshape(-1)
    if np.any((cnt > 0) & ((st < 0) | (st + cnt > len(neighbours)))):
        raise GridFileError("neighbour list outside the neighbour array")
    return d, energrads, neighbours, cnt, st, big, potentials


def read_grid_csr(grid_data: bytes, read_gradients: bool = True):
    """``(fields, nb_hdr [V,2] {start, count}, nb_list u16)``: the grid with its
    neighbour lists in CSR form (V = dx*dy*dz points, x slowest, as the kernels
    index them); ``fields`` holds every ``read_grid`` field but the padded
    neighbour grid."""
    d, energrads, neighbours, cnt, st, big, potentials = _parse(grid_data, read_gradients)
    off = np.cumsum(cnt) - cnt
    total = int(cnt.sum())
    rows = np.repeat(np.arange(len(cnt)), cnt)
    k = np.arange(total) - np.repeat(off, cnt)
    nb_list = neighbours[st[rows] + k].astype(np.uint16)
    d["max_nr_neighbours"] = d["nr_neighbours"].max() if d["nr_neighbours"].size else 0
    if big is not None:
        d["outer_potential_grid"] = potentials(big, tuple(int(v) for v in d["dim2"]), True)
    return d, np.stack([off, cnt], 1), nb_list


def read_grid(grid_data: bytes, read_gradients: bool = False):
    """The reference's ``read_grid`` (read_grid2.py:16-161): same fields, same
    arrays (``neighbour_grid [dx,dy,dz,max_nr_neighbours]`` uint16 padded with
    65535), same errors for unsupported grids (raised as :class:`GridFileError`)."""
    d, nb_hdr, nb_list = read_grid_csr(grid_data, read_gradients)
    dx, dy, dz = (int(v) for v in d["dim"])
    maxnb = int(max(d["max_nr_neighbours"], 0))
    ng = np.full((dx * dy * dz, maxnb), 2 ** 16 - 1, np.uint16)
    off, cnt = nb_hdr[:, 0], nb_hdr[:, 1]
    rows = np.repeat(np.arange(len(cnt)), cnt)
    ng[rows, np.arange(len(nb_list)) - np.repeat(off, cnt)] = nb_list
    d["neighbour_grid"] = ng.reshape(dx, dy, dz, maxnb)
    d["max_nr_neighbours"] = d["nr_neighbours"].max()
    # a grid without potentials has no inner/outer fields (read_grid2.py:159)
    keys = [f for f in GRID_FIELDS[:-1] if f in d]
    cls = GridTuple if len(keys) == len(GRID_FIELDS) - 1 else namedtuple("Grid", keys + ["neighbour_grid_ravel"])
    return cls(*[d[k] for k in keys], None)


def write_grid(*, gridspacing, gridextension, plateaudis, neighbourdis, alphabet, origin, dim, dim2, natoms,
               inner_potential_grid=None, outer_potential_grid=None, nb_hdr=None, nb_list=None,
               neighbour_grid=None, nr_neighbours=None, rec_type=None, pivot=(0.0, 0.0, 0.0)) -> bytes:
    """ATTRACT ``.grid`` bytes for dense grids ``[T, x, y, z, 4]`` (T = the
    number of true entries of ``alphabet``) and a neighbour grid given as CSR
    (``nb_hdr``/``nb_list``, points x slowest) or dense (``neighbour_grid`` +
    ``nr_neighbours``).  Every inner value gets its own energrad entry; an outer
    point whose 4 values are all zero is written as "no value" (index 0)."""
    alphabet = np.asarray(alphabet, bool).reshape(-1)
    if alphabet.shape != (99,):
        raise ValueError("alphabet must have 99 entries")
    dx, dy, dz = (int(v) for v in dim)
    dx2, dy2, dz2 = (int(v) for v in dim2)
    V = dx * dy * dz
    present = np.flatnonzero(alphabet)
    T = len(present)
    parts = [_HEAD.pack(False, 64, float(gridspacing), int(gridextension), float(plateaudis), float(neighbourdis),
                        *[bool(a) for a in alphabet], *[float(v) for v in origin], dx, dy, dz, dx2, dy2, dz2,
                        int(natoms), *[float(v) for v in pivot])]
    file_order = lambda a: np.ascontiguousarray(np.moveaxis(a, (1, 2, 3), (3, 2, 1)))  # [T, z, y, x, ...]
    energrads = []
    pot_inner = np.zeros((V, 100), np.uint32)
    pot_outer = None
    n = 0
    if inner_potential_grid is not None:
        g = np.asarray(inner_potential_grid, np.float32)
        if g.shape != (T, dx, dy, dz, 4):
            raise ValueError(f"inner grid shape {g.shape} != {(T, dx, dy, dz, 4)}")
        energrads.append(file_order(g).reshape(T * V, 4))
        pot_inner[:, present] = (1 + np.arange(T * V, dtype=np.int64).reshape(T, V)).T
        n = T * V
        pot_outer = np.zeros((dx2 * dy2 * dz2, 100), np.uint32)
        if outer_potential_grid is not None:
            go = np.asarray(outer_potential_grid, np.float32)
            if go.shape != (T, dx2, dy2, dz2, 4):
                raise ValueError(f"outer grid shape {go.shape} != {(T, dx2, dy2, dz2, 4)}")
            vals = file_order(go).reshape(T, -1, 4)
            keep = np.any(vals != 0, axis=2)
            idx = np.zeros(keep.shape, np.int64)
            idx[keep] = n + 1 + np.arange(int(keep.sum()))
            energrads.append(vals[keep])
            pot_outer[:, present] = idx.T
            n += int(keep.sum())
    eg = np.concatenate(energrads) if energrads else np.zeros((0, 4), np.float32)
    parts.append(struct.pack("=2i", len(eg), -1))
    parts.append(eg.astype(np.float32).tobytes())
    if neighbour_grid is not None:
        ngr = np.asarray(neighbour_grid).reshape(V, -1)
        cnt = np.clip(np.asarray(nr_neighbours, np.int64).reshape(-1), 0, ngr.shape[1])
        mask = np.arange(ngr.shape[1])[None, :] < cnt[:, None]
        nb_list = ngr[mask]
        nb_hdr = np.stack([np.cumsum(cnt) - cnt, cnt], 1)
    if nb_hdr is None:
        nb_hdr = np.zeros((V, 2), np.int64)
        nb_list = np.zeros(0, np.uint16)
    nb_hdr = np.asarray(nb_hdr, np.int64).reshape(V, 2)
    nb_list = np.asarray(nb_list).reshape(-1)
    cnt = nb_hdr[:, 1]
    # the neighbour array in point order of the file (x fastest)
    to_file = lambda a: np.ascontiguousarray(a.reshape(dx, dy, dz).transpose(2, 1, 0)).reshape(-1)
    cnt_f = to_file(cnt)
    start_f = to_file(nb_hdr[:, 0])
    rows = np.repeat(np.arange(V), cnt_f)
    k = np.arange(int(cnt_f.sum())) - np.repeat(np.cumsum(cnt_f) - cnt_f, cnt_f)
    entries = nb_list[start_f[rows] + k].astype(np.uint32) if len(rows) else np.zeros(0, np.uint32)
    nb = np.zeros(len(entries), _NB_DTYPE)
    nb["index"] = entries
    if rec_type is not None and len(entries):
        nb["type"] = np.asarray(rec_type, np.int64)[entries].astype(np.uint8)
    parts.append(struct.pack("=2i", len(nb), -1))
    parts.append(nb.tobytes())
    inner = np.zeros(V, _INNER_DTYPE)
    inner["potential"] = pot_inner  # rows already in file point order
    inner["neighbourlist"] = np.where(cnt_f > 0, np.cumsum(cnt_f) - cnt_f + 1, 0)
    nr = to_file(np.asarray(nr_neighbours, np.int64).reshape(-1)) if nr_neighbours is not None else cnt_f
    inner["nr_neighbours"] = nr.astype(np.int16)
    parts.append(struct.pack("=q", V))
    parts.append(inner.tobytes())
    if pot_outer is not None:
        parts.append(struct.pack("=q", dx2 * dy2 * dz2))
        parts.append(pot_outer.tobytes())
    else:
        parts.append(struct.pack("=q", 0))
    return b"".join(parts)
