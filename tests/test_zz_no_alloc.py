"""att_nbgrid_count_noalloc -- the neighbour-list count without a caller
workspace -- against att_nbgrid_count, both through the C ABI.

Some callers cannot allocate device memory: a plugin that only gets the
buffers of a host framework whose allocator owns all GPU memory, an FFI
binding without an allocator of its own, or a service that must never call
cudaMalloc/cudaFree because they synchronise the device.  They call the
no-allocation entry point, which keeps its scan workspace in a fixed array
inside the library.  This file is collected last, so that a run stopping at
the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _lib():
    from attract_b200 import _lib

    return _lib, _lib.load()


def _geom(dims, origin, spacing=0.9):
    from attract_b200 import GridGeom

    return GridGeom(tuple(origin), spacing, tuple(dims), (2, 2, 2), 0, 5.0, 1).to_c()


def _receptor(n, seed):
    from attract_b200 import synth
    from attract_b200.grid import pack_receptor

    xyz, t, R = synth.receptor_beads(n, seed=seed)
    return pack_receptor(xyz, t, torch.device("cuda")), n


def _count(L, lib, gc, rec, n_rec, radius, noalloc):
    nvox = gc.dim[0] * gc.dim[1] * gc.dim[2]
    hdr = torch.full((nvox, 2), -7, dtype=torch.int32, device="cuda")
    total = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    if noalloc:
        rc = lib.att_nbgrid_count_noalloc(C.byref(gc), rec.data_ptr(), n_rec, radius, hdr.data_ptr(),
                                          total.data_ptr(), st)
        L.check(rc, "att_nbgrid_count_noalloc")
    else:
        wsb = lib.att_nbgrid_workspace_bytes(nvox)
        ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
        rc = lib.att_nbgrid_count(C.byref(gc), rec.data_ptr(), n_rec, radius, hdr.data_ptr(), total.data_ptr(),
                                  ws.data_ptr(), wsb, st)
        L.check(rc, "att_nbgrid_count")
    torch.cuda.synchronize()
    return hdr.cpu().numpy(), int(total.item())


def test_noalloc_count_matches_workspace_count_on_consecutive_calls():
    """Two calls in a row (a large grid, then a smaller one that leaves stale
    words of the first call in the shared array) give the same headers and
    totals as the entry point with a caller workspace."""
    L, lib = _lib()
    cases = [((130, 124, 118), (-58.0, -55.0, -52.0), 2500, 1),   # 1.9 M points: multi-chunk block scan
             ((61, 57, 49), (-27.0, -25.0, -22.0), 600, 2)]
    for dims, origin, n, seed in cases:
        rec, n_rec = _receptor(n, seed)
        gc = _geom(dims, origin)
        radius = 5.0 + 0.9 * np.sqrt(3) / 2
        h1, t1 = _count(L, lib, gc, rec, n_rec, radius, noalloc=True)
        h0, t0 = _count(L, lib, gc, rec, n_rec, radius, noalloc=False)
        assert t1 == t0 and t0 > 0
        assert np.array_equal(h1, h0)
        assert h1[:, 1].sum() == t1


def test_noalloc_rejects_grids_beyond_the_fixed_workspace():
    L, lib = _lib()
    rec, n_rec = _receptor(50, 3)
    gc = _geom((256, 256, 129), (0.0, 0.0, 0.0))  # 8.45 M points > 8 M
    hdr = torch.zeros(2, dtype=torch.int32, device="cuda")
    total = torch.zeros(1, dtype=torch.int64, device="cuda")
    rc = lib.att_nbgrid_count_noalloc(C.byref(gc), rec.data_ptr(), n_rec, 5.0, hdr.data_ptr(), total.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream)
    assert rc == 1
    assert b"fixed workspace" in lib.att_last_error_string()


def test_noalloc_count_at_exactly_the_maximum_grid():
    """A grid of exactly ATT_NBGRID_NOALLOC_MAX_VOXELS points (256 x 256 x 128),
    where the count kernel writes the last word of the fixed array, equals the
    entry point with a caller workspace."""
    L, lib = _lib()
    rec, n_rec = _receptor(400, 4)
    gc = _geom((256, 256, 128), (-60.0, -60.0, -30.0), spacing=0.47)
    assert gc.dim[0] * gc.dim[1] * gc.dim[2] == 8192 * 1024
    h1, t1 = _count(L, lib, gc, rec, n_rec, 5.0, noalloc=True)
    h0, t0 = _count(L, lib, gc, rec, n_rec, 5.0, noalloc=False)
    assert t1 == t0 and t0 > 0
    assert np.array_equal(h1, h0)
