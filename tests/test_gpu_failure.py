"""Failure paths on the GPU without faulting it.  The kernels hold no wait
that another thread or a flag must end (a lane waits only for its own
cp.async copies), so no wait can time out.  Non-finite inputs are flagged per
pose, never trapped; caller tables that point outside their arrays are
refused per pose before any access, with ATT_KERR_BAD_SEGMENT in the device
error word."""
import numpy as np
import pytest
import torch

from gpu_cases import small_case, to_device_grid

pytestmark = pytest.mark.gpu


def _case(n_poses=64):
    import attract_b200 as A

    A.load_library()
    c = small_case(seed=90, n_poses=n_poses)
    grid = to_device_grid(c)
    wl = A.Workload([grid], A.LigandSet([(c["lig"], c["gt"], c["lt"])]), [A.Segment(0, 0, n_poses)],
                    lanes_per_pose=32)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    return A, c, wl, P


def test_reserved_test_flags_are_rejected():
    """AttLaunchCfg.test_flags is reserved: a non-zero value is an argument
    error, answered before any launch."""
    A, c, wl, P = _case(n_poses=8)
    with pytest.raises(A.AttractError, match="reserved"):
        A.minimise(wl, P, 2, launch=A.LaunchShape(32, test_flags=1))


def test_nonfinite_poses_are_flagged_not_trapped():
    A, c, wl, P = _case(n_poses=32)
    bad = P.clone()
    bad[3, 4] = float("nan")
    bad[7, 0] = float("inf")
    out, E, S, _ = A.minimise(wl, bad, 3)
    S = S.cpu().numpy()
    from attract_b200 import _lib

    assert S[3] & _lib.ATT_STATUS_NONFINITE_POSE and S[7] & _lib.ATT_STATUS_NONFINITE_POSE
    ok = np.ones(32, bool)
    ok[[3, 7]] = False
    assert np.all(S[ok] == 0)
    assert np.all(np.isfinite(E.cpu().numpy()[ok]))
    E2, G2, S2 = A.energrad(wl, bad)
    assert S2.cpu().numpy()[3] & _lib.ATT_STATUS_NONFINITE_POSE
    mats = torch.zeros((32, 16), dtype=torch.float32, device="cuda")
    mats[:, [0, 5, 10, 15]] = 1.0
    mats[5, 13] = float("nan")
    _, _, S3 = A.energrad(wl, mats)
    S3 = S3.cpu().numpy()
    assert S3[5] & _lib.ATT_STATUS_NONFINITE_POSE and S3[4] == 0


def _raw_energrad(A, wl, segs, P, pose_lig=None, n_rows=None):
    """att_energrad through the C ABI with a caller-made segment table (the
    host-side checks of the Python layer are bypassed on purpose)."""
    import ctypes as C

    from attract_b200 import _lib

    B = wl.n_poses if n_rows is None else n_rows
    E = torch.full((B,), float("nan"), dtype=torch.float32, device="cuda")
    G = torch.full((B, 6), float("nan"), dtype=torch.float32, device="cuda")
    S = torch.full((B,), -1, dtype=torch.int32, device="cuda")
    cfg = A.EvalOptions().to_c(0)
    lc = A.LaunchShape(wl.lanes).to_c()
    rc = _lib.load().att_energrad(wl.c_grids, len(wl.grids), C.byref(wl.c_ligs), segs.data_ptr(), segs.shape[0],
                                  wl.seg_tile.data_ptr(), wl.n_tiles, B, P.data_ptr(), _lib.ptr(pose_lig),
                                  C.byref(cfg), E.data_ptr(), G.data_ptr(), S.data_ptr(), C.byref(lc),
                                  torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "att_energrad")
    torch.cuda.synchronize()
    return E.cpu().numpy(), G.cpu().numpy(), S.cpu().numpy()


@pytest.mark.parametrize("lanes", [8, 32])
def test_bad_segments_are_skipped_before_any_access(lanes):
    """A C caller's segment table that names a missing grid or ligand, or
    reaches beyond the pose arrays, and conformer indices that leave the
    ligand set (the reference asserts every such index, test5.py:55-61,79-82,
    90,98): the kernel checks them before any access, skips those poses
    (outputs unwritten), sets ATT_KERR_BAD_SEGMENT, and every other pose's
    result is bit-identical to a launch of the valid segments."""
    import attract_b200 as A
    from attract_b200 import _lib

    A.load_library()
    c = small_case(seed=91, n_poses=48)
    grid = to_device_grid(c)
    ligs = A.LigandSet([(c["lig"], c["gt"], c["lt"])])
    wl = A.Workload([grid], ligs, [A.Segment(0, 0, 16)] * 3, lanes_per_pose=lanes)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    E_ref, G_ref, S_ref = _raw_energrad(A, wl, wl.segs, P)
    assert _lib.kernel_status(clear=True) == 0
    assert np.all(np.isfinite(E_ref)) and np.all(S_ref == 0)
    keep = np.r_[0:16, 32:48]
    for field, value in (("grid", 5), ("grid", -1), ("lig", 1), ("pose0", 40), ("n_poses", 40), ("pose0", -8)):
        segs = wl.segs.clone()
        segs[1, ("grid", "lig", "pose0", "n_poses").index(field)] = value
        E, G, S = _raw_energrad(A, wl, segs, P)
        word = _lib.kernel_status(clear=True)
        assert word & _lib.ATT_KERR_BAD_SEGMENT, (field, value, word)
        assert np.array_equal(E[keep], E_ref[keep]) and np.array_equal(G[keep], G_ref[keep]), (field, value)
        assert np.all(np.isnan(E[16:32])) and np.all(S[16:32] == -1), (field, value)
    # conformer indices: pose 20's index leaves the ligand set, the rest are 0
    pl = torch.zeros(48, dtype=torch.int32, device="cuda")
    pl[20] = 3
    E, G, S = _raw_energrad(A, wl, wl.segs, P, pose_lig=pl)
    assert _lib.kernel_status(clear=True) & _lib.ATT_KERR_BAD_SEGMENT
    others = np.r_[0:20, 21:48]
    assert np.isnan(E[20]) and S[20] == -1
    assert np.array_equal(E[others], E_ref[others])
    # pose arrays declared shorter than the segments need: the last segment is refused
    E, G, S = _raw_energrad(A, wl, wl.segs, P, n_rows=40)
    assert _lib.kernel_status(clear=True) & _lib.ATT_KERR_BAD_SEGMENT
    assert np.array_equal(E[:32], E_ref[:32]) and np.all(np.isnan(E[32:40]))
    # and a clean launch afterwards leaves the word at 0
    E, _, _ = _raw_energrad(A, wl, wl.segs, P)
    assert _lib.kernel_status(clear=True) == 0 and np.array_equal(E, E_ref)
