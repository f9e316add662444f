"""Host-side logic and the C-ABI library (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import attract_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "attract_b200.h")


def _lib_path():
    from attract_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        from attract_b200 import build

        build.build()
    return _lib.LIB_PATH


def test_library_exports_every_declared_symbol():
    from attract_b200 import _lib

    text = open(HEADER).read()
    declared = set(re.findall(r"\b(att_[a-z0-9_]+)\s*\(", text))
    assert declared, "no declarations found"
    lib = C.CDLL(_lib_path())
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_lib.SIGNATURES), declared ^ set(_lib.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", _lib_path()], capture_output=True, text=True).stdout
    for name in declared:
        assert re.search(rf"\bT {name}$", out, re.M), name


def test_ctypes_layouts_match_the_c_header(tmp_path):
    from attract_b200 import _lib

    src = tmp_path / "probe.c"
    structs = ["AttGridGeom", "AttGrid", "AttLigands", "AttSegment", "AttEvalCfg", "AttAdamCfg", "AttLaunchCfg",
               "AttSchemaCfg"]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "attract_b200.h"', "int main(void){"]
    for s in structs:
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f, _ in getattr(_lib, s)._fields_:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for s in structs:
        cls = getattr(_lib, s)
        assert int(got[s]) == C.sizeof(cls), s
        for f, _ in cls._fields_:
            assert int(got[f"{s}.{f}"]) == getattr(cls, f).offset, f"{s}.{f}"


def test_error_path_without_gpu():
    """Argument validation answers before any CUDA call."""
    from attract_b200 import _lib

    lib = _lib.load(_lib_path())
    rc = lib.att_energrad(None, 0, None, None, 0, None, 0, 0, None, None, None, None, None, None, None, None)
    assert rc == 1
    assert b"n_grids" in lib.att_last_error_string()
    g = _lib.AttGridGeom()
    assert lib.att_grid_brick_bytes(C.byref(g), 1) == -1
    g.dim[:] = [3, 3, 3]
    g.dim2[:] = [3, 3, 3]
    g.spacing = 1.0
    g.n_types = 2
    assert lib.att_grid_brick_bytes(C.byref(g), 1) == 2 * (8 + 8) * 128
    assert lib.att_grid_brick_bytes(C.byref(g), 0) == 2 * 8 * 128
    assert lib.att_nbgrid_workspace_bytes(5000) >= 4 * 5


def test_forcefield_pair_table_matches_oracle():
    from attract_b200 import ForceField

    ff = ForceField.synthetic(6, seed=3)
    for shift in (True, False):
        t = ff.pair_table(5.0, shift)
        ref = O.pair_table(ff.rc, ff.ac, ff.ivor, 5.0, shift, ff.rcap2)
        assert np.allclose(t, ref, rtol=1e-6, atol=0)


def test_forcefield_from_attract_par_roundtrip(golden):
    from attract_b200 import ForceField

    rbc, abc, ipon = golden["par15"]
    # a 2-type par file with the 15-15 entry on the diagonal
    txt = "8 2 0 0\n" + "\n".join(" ".join(f"{v:.2f}" for v in row) for row in
                                  ([rbc, 3.0], [3.0, rbc], [abc, 1.0], [1.0, abc], [ipon, -1], [-1, ipon]))
    ff = ForceField.from_attract_par(txt)
    assert np.isclose(ff.rc[0, 0], abc * rbc ** 8) and ff.ivor[0, 1] == -1
    rc, ac, iv = O.ff_from_attract_par(txt)
    assert np.allclose(ff.rc, rc) and np.allclose(ff.ac, ac) and np.array_equal(ff.ivor, iv)


def test_pose_conventions_match_oracle():
    from attract_b200 import poses as P

    rng = np.random.default_rng(0)
    p = np.concatenate([rng.uniform(-3, 3, (40, 3)), rng.normal(size=(40, 3))], 1)
    assert np.allclose(P.pose_to_mat(p), O.pose_to_mat(p))
    assert np.allclose(P.pose_to_mat(P.mat_to_pose(P.pose_to_mat(p))), P.pose_to_mat(p), atol=1e-12)
    rot = P.random_rotations(2000, rng)
    Q = P.euler_to_Q(*rot.T)
    assert np.allclose(np.einsum("bij,bkj->bik", Q, Q), np.eye(3), atol=1e-12)
    # uniform on SO(3): the mean rotation matrix vanishes
    assert np.abs(Q.mean(0)).max() < 0.05


def test_synthetic_receptor_separation_and_density():
    from attract_b200 import synth

    xyz, t, R = synth.receptor_beads(400, radius=20.0, seed=2)
    from scipy.spatial import cKDTree

    d, _ = cKDTree(xyz).query(xyz, 2)
    assert d[:, 1].min() >= 3.5 - 1e-9
    assert np.linalg.norm(xyz, axis=1).max() <= 20.0
    assert t.min() >= 0 and t.max() < 32
    _, _, R6 = synth.receptor_beads(600, seed=3)  # default: 40 A sphere
    assert R6 == 40.0


def test_workload_tiling_on_cpu():
    from attract_b200 import ForceField, Grid, GridGeom, LigandSet, Segment, Workload

    ff = ForceField.synthetic(4, 0)
    geom = GridGeom((0, 0, 0), 1.0, (4, 4, 4), (3, 3, 3), 1, 2.0, 4)
    g = Grid(geom, np.zeros((2, 3)), [0, 1], ff, device="cpu")
    L = LigandSet([(np.zeros((3, 3)), [0, 1, 2], None), (np.zeros((5, 3)), [0] * 5, None)], device="cpu")
    wl = Workload([g], L, [Segment(0, 0, 9), Segment(0, 1, 0), Segment(0, 1, 4)], lanes_per_pose=8)
    assert wl.seg_tile.tolist() == [0, 3, 3, 4]
    assert wl.n_tiles == 4 and wl.n_poses == 13
    assert wl.segs[:, 2].tolist() == [0, 9, 9]
    wl32 = wl.with_lanes(32)
    assert wl32.seg_tile.tolist() == [0, 9, 9, 13]
    with pytest.raises(ValueError):
        Workload([g], L, [Segment(0, 2, 1)])
    with pytest.raises(ValueError):
        LigandSet([(np.zeros((2, 3)), [0, 70000], None)], device="cpu")


def test_serving_launch_shapes():
    """A request's launch shape follows its own ligand size: beads per lane
    as the kernel picks them (next power of two, at most 4)."""
    from attract_b200.serve import launch_shape

    assert launch_shape(1, 32) == (32, 1) and launch_shape(32, 32) == (32, 1)
    assert launch_shape(33, 32) == (32, 2) and launch_shape(64, 32) == (32, 2)
    assert launch_shape(65, 32) == (32, 4) and launch_shape(500, 32) == (32, 4)
    assert launch_shape(9, 8) == (8, 2) and launch_shape(17, 8) == (8, 4) and launch_shape(16, 16) == (16, 1)
    for bad in ((10, 12), (0, 32)):
        with pytest.raises(ValueError):
            launch_shape(*bad)


def test_attract_par_errors_are_clear():
    from attract_b200 import ForceField

    good = "8 2\n" + " ".join(["1.0"] * 12)
    ff = ForceField.from_attract_par(good)
    assert ff.rc.shape == (2, 2)
    for text, msg in (("", "first line"), ("7 2\n1", "potshape"), ("8 0\n", "types"),
                      ("8 2\n" + " ".join(["1.0"] * 11), "values")):
        with pytest.raises(ValueError, match=msg):
            ForceField.from_attract_par(text)
    with pytest.raises(ValueError, match="outside"):
        ForceField.from_attract_par(good, rec_types=[1, 3])


def test_invalid_geometry_is_rejected_by_both_count_entry_points():
    """att_nbgrid_count and att_nbgrid_count_noalloc take the same arguments
    and apply the same geometry rules (validation answers before any CUDA
    call, so this runs without a GPU)."""
    from attract_b200 import _lib

    lib = _lib.load(_lib_path())
    bad = []
    for field, value in (("dim", [1, 4, 4]), ("dim2", [-1, 2, 2]), ("spacing", 0.0), ("plateau", -1.0),
                         ("n_types", 0)):
        g = _lib.AttGridGeom()
        g.dim[:] = [4, 4, 4]
        g.dim2[:] = [2, 2, 2]
        g.spacing, g.plateau, g.n_types = 1.0, 3.0, 1
        if isinstance(value, list):
            getattr(g, field)[:] = value
        else:
            setattr(g, field, value)
        bad.append(g)
    for g in bad:
        rc0 = lib.att_nbgrid_count(C.byref(g), None, 0, 1.0, None, None, None, 0, None)
        msg0 = lib.att_last_error_string()
        rc1 = lib.att_nbgrid_count_noalloc(C.byref(g), None, 0, 1.0, None, None, None)
        msg1 = lib.att_last_error_string()
        assert rc0 == rc1 == 1, (rc0, rc1)
        assert msg0 == msg1, (msg0, msg1)


def test_list_total_beyond_32_bit_starts_is_rejected():
    """The CSR starts are 32-bit: a neighbour grid whose entry total does not
    fit is refused before the lists are allocated or filled."""
    from attract_b200 import grid

    grid.check_list_total(0)
    grid.check_list_total(2 ** 32 - 1)
    with pytest.raises(ValueError, match="32-bit"):
        grid.check_list_total(2 ** 32)
