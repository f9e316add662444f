"""Explicit all-pairs rescoring (att_allpairs_energy) against ATTRACT's own
scores (mono-leu minim-sorted.score, --rcut 9999999) and the oracle.

Tolerances (float32 kernel, float64 references): energy |dE| <= 1e-5 * S_E +
1e-3, S_E = sum of |pair energy| (float32 summation error is bounded by the sum
of magnitudes); gradient |dg| <= 1e-4 * S_g + 1e-3 with S_g = sum of |pair
gradient| (1 + |lever arm|)."""
import numpy as np
import pytest
import torch

import attract_oracle as O
from conftest import dat_poses
from gpu_cases import small_case

pytestmark = pytest.mark.gpu


def _ff15(golden):
    from attract_b200 import ForceField

    rbc, abc, ipon = golden["par15"]
    return ForceField([[abc * rbc ** 8]], [[abc * rbc ** 6]], [[ipon]])


def test_mono_leu_matches_attract_scores(golden):
    from attract_b200 import load_library
    from attract_b200.allpairs import AllPairs

    load_library()
    beads = golden["beads"]
    n = len(beads)
    pose = dat_poses(golden)
    ff = _ff15(golden)
    ap = AllPairs(beads, np.zeros(n, int), beads, np.zeros(n, int), ff)
    E, G = ap.energy(torch.tensor(pose, dtype=torch.float32, device="cuda"), grad=True)
    E = E.cpu().numpy()
    ref = golden["score_allpairs"][: len(pose)]
    sub = slice(0, 12)  # the oracle pass over 1.6 M pairs per pose: a subset
    pair = O.pair_table(ff.rc, ff.ac, ff.ivor, 5.0, shift_plateau=False)
    Eo, Go, ea, ga = O.allpairs_energrad(pose[sub], beads, np.zeros(n, int), beads, np.zeros(n, int), pair)
    assert np.all(np.abs(E[sub] - Eo) <= 1e-5 * ea + 1e-3)
    assert np.all(np.abs(G.cpu().numpy()[sub] - Go) <= 1e-4 * ga[:, None] + 1e-3)
    # every pose against ATTRACT; the oracle itself agrees with ATTRACT to 1e-7 of max |E|
    scale = np.abs(ref).max()
    assert np.all(np.abs(E - ref) <= 2e-5 * scale), np.abs(E - ref).max() / scale


@pytest.mark.parametrize("rcut", [0.0, 6.0])
def test_synthetic_types_cutoff_and_gradients(rcut):
    from attract_b200 import ForceField, load_library
    from attract_b200.allpairs import AllPairs

    load_library()
    c = small_case(seed=70, n_poses=48, ivor_mix=True)  # capped, mixed ivor
    G = c["G"]
    ff = ForceField(c["rc"], c["ac"], c["ivor"], c["rcap2"])
    ap = AllPairs(G["rec"], G["rtype"], c["lig"], c["lt"], ff)
    poses = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    E, Gr = ap.energy(poses, rcut=rcut or None, grad=True)
    pair = O.pair_table(c["rc"], c["ac"], c["ivor"], 1.0, shift_plateau=False, rcap2=c["rcap2"])
    Eo, Go, ea, ga, gb = O.allpairs_energrad(c["poses"], c["lig"], c["lt"], G["rec"], G["rtype"], pair,
                                             rcut2=rcut * rcut if rcut else None, bead_grad=True)
    assert np.all(np.abs(E.cpu().numpy() - Eo) <= 1e-5 * ea + 1e-4)
    assert np.all(np.abs(Gr.cpu().numpy() - Go) <= 1e-4 * ga[:, None] + 1e-3)
    # the 4x4 form: same energies; dE/dM[r][c] = sum_b x_r g_c, dE/dt = sum_b g_b (test1.py:409-412)
    mats = torch.tensor(O.pose_to_mat(c["poses"]), dtype=torch.float32, device="cuda")
    Em, Gm = ap.energy(mats, rcut=rcut or None, grad=True)
    Gm = Gm.cpu().numpy()
    assert np.all(np.abs(Em.cpu().numpy() - Eo) <= 1e-5 * ea + 1e-4)
    dM = np.einsum("nr,bnc->brc", c["lig"], gb)
    assert np.all(np.abs(Gm[:, :3, :3] - dM) <= 1e-4 * ga[:, None, None] + 1e-3)
    assert np.all(np.abs(Gm[:, 3, :3] - gb.sum(1)) <= 1e-4 * ga[:, None] + 1e-3)
    assert np.all(Gm[:, :, 3] == 0)


def test_rejects_bad_arguments():
    from attract_b200 import AttractError, ForceField, load_library
    from attract_b200 import _lib

    load_library()
    lib = _lib.load()
    with pytest.raises(AttractError):
        _lib.check(lib.att_allpairs_energy(None, 0, None, 0, None, 1, 0, None, 1, 1, 0.0, None, None, None),
                   "att_allpairs_energy")
    with pytest.raises(ValueError):
        from attract_b200.allpairs import AllPairs

        AllPairs(np.zeros((2, 3)), [0, 5], np.zeros((1, 3)), [0], ForceField([[1.0]], [[1.0]], [[1.0]]))
