"""Failure paths on the GPU without faulting it: a copy wait that never
completes (a 16-byte expectation no copy delivers, injected on request) runs
out after about a second, the kernel reports ATT_KERR_COPY_TIMEOUT in the
device error word and returns, and the context stays usable.  Non-finite
inputs are flagged per pose, never trapped."""
import time

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


def test_stalled_copy_wait_times_out_and_the_context_survives():
    from attract_b200 import _lib

    A, c, wl, P = _case()
    ref_out, ref_E, _, _ = A.minimise(wl, P, 4)
    ref_out, ref_E = ref_out.clone(), ref_E.clone()
    assert _lib.kernel_status(clear=True) == 0
    t0 = time.perf_counter()
    A.minimise(wl, P, 4, launch=A.LaunchShape(32, test_flags=_lib.ATT_TEST_STALL_COPY_WAIT))
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    word = _lib.kernel_status(clear=True)
    assert word & _lib.ATT_KERR_COPY_TIMEOUT, word
    assert 0.5 < dt < 60.0, dt  # the bounded wait: about a second
    assert _lib.kernel_status(clear=True) == 0  # cleared
    # the same launch without the hook still gives the reference result
    out, E, S, _ = A.minimise(wl, P, 4)
    assert torch.equal(out, ref_out) and torch.equal(E, ref_E)
    assert _lib.kernel_status(clear=True) == 0


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
