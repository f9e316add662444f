"""The oracle against the reference's golden vectors (CPU only)."""
import numpy as np
import pytest
from hypothesis import given, settings
from hypothesis import strategies as st

import attract_oracle as O
from conftest import dat_poses, mono_leu_setup


def _ff15(g):
    rbc, abc, ipon = g["par15"]
    rc, ac = abc * rbc ** 8, abc * rbc ** 6
    emin = -27.0 * ac ** 4 / (256.0 * rc ** 3)
    rmin2 = 4.0 * rc / (3.0 * ac)
    return rc, ac, emin, rmin2, float(ipon)


def test_par15_matches_energy_init_constants(golden):
    # energy-init/energy-init.py:1-3 hard-codes the 15-15 entry of attract.par
    assert np.allclose(golden["par15"], [3.88, 13.81, 1.0])


def test_nonbon_vs_attract_energy_init(golden):
    rc, ac, emin, rmin2, iv = _ff15(golden)
    d = golden["pair_dist"]
    e = O.nonbon(d * d, rc, ac, emin, rmin2, iv)
    ref = golden["pair_energy_attract"]
    rel = np.abs(e - ref) / np.maximum(np.abs(ref), 1e-3)
    assert rel.max() < 1e-5, rel.max()  # ATTRACT prints ~17 digits; distances carry ~16


def test_dnonbon_is_derivative(golden):
    rc, ac, emin, rmin2, iv = _ff15(golden)
    for ivor in (1.0, -1.0):
        dsq = np.linspace(4.0, 60.0, 500)
        h = 1e-6
        fd = (O.nonbon(dsq + h, rc, ac, emin, rmin2, ivor) - O.nonbon(dsq - h, rc, ac, emin, rmin2, ivor)) / (2 * h)
        an = O.dnonbon_ddsq(dsq, rc, ac, emin, rmin2, ivor)
        ok = np.abs(dsq - rmin2) > 1e-3
        assert np.allclose(fd[ok], an[ok], rtol=1e-5, atol=1e-9)


def test_euler_convention_vs_reference_matrices(golden):
    pose = dat_poses(golden)
    mat = O.pose_to_mat(pose[:4])
    ref = golden["mat10"][:4]
    assert np.abs(mat[:, :3, :3] - ref[:, :3, :3]).max() < 1e-6
    assert np.abs(mat[:, 3, :3] - ref[:, 3, :3]).max() < 1e-9
    back = O.mat_to_euler(mat)
    assert np.allclose(O.pose_to_mat(back), mat, atol=1e-12)


def test_euler_matches_scipy_zyz(golden):
    from scipy.spatial.transform import Rotation

    rng = np.random.default_rng(1)
    a = rng.uniform(-np.pi, np.pi, (50, 3))
    M = Rotation.from_euler("zyz", np.stack([-a[:, 0], -a[:, 1], a[:, 2]], 1)).as_matrix()
    assert np.allclose(O.pose_to_mat(np.concatenate([a, np.zeros((50, 3))], 1))[:, :3, :3], M, atol=1e-12)


def test_euler_axes_are_derivatives():
    rng = np.random.default_rng(2)
    a = rng.uniform(-3, 3, (20, 3))
    Q = O.euler_to_Q(a[:, 0], a[:, 1], a[:, 2])
    W = O.euler_axes(a[:, 0], a[:, 1])
    h = 1e-6
    for k in range(3):
        ap, am = a.copy(), a.copy()
        ap[:, k] += h
        am[:, k] -= h
        dQ = (O.euler_to_Q(*ap.T) - O.euler_to_Q(*am.T)) / (2 * h)
        w = W[:, k]
        cross = np.zeros((20, 3, 3))
        cross[:, 0, 1], cross[:, 0, 2], cross[:, 1, 2] = -w[:, 2], w[:, 1], -w[:, 0]
        cross[:, 1, 0], cross[:, 2, 0], cross[:, 2, 1] = w[:, 2], -w[:, 1], w[:, 0]
        assert np.allclose(dQ, cross @ Q, atol=1e-8)


def test_allpairs_vs_attract_score(golden):
    pose = dat_poses(golden)[:8]
    rc, ac, emin, rmin2, iv = _ff15(golden)
    pair = O.pair_table([[rc]], [[ac]], [[iv]], 5.0, shift_plateau=False)
    beads = golden["beads"]
    E = O.allpairs_energy(pose, beads, np.zeros(len(beads), int), beads, np.zeros(len(beads), int), pair)
    ref = golden["score_allpairs"][:8]
    assert np.abs(E - ref).max() / np.abs(ref).max() < 1e-7


@pytest.fixture(scope="module")
def nb_plain(golden):
    return mono_leu_setup(golden, shift_plateau=False)


@pytest.fixture(scope="module")
def nb_plat(golden):
    return mono_leu_setup(golden, shift_plateau=True)


def _lig(g):
    n = len(g["beads"])
    return g["beads"], np.zeros(n, int), np.zeros(n, int)


def test_nb_plain_vs_attract_nbgrid_score(golden, nb_plain):
    pose = dat_poses(golden)[:16]
    lig, gt, lt = _lig(golden)
    E, grad = O.energrad(pose, lig, gt, lt, nb_plain)
    refE = golden["score_nbgrid_energy"][:16]
    refG = golden["score_nbgrid_grad"][:16]  # ATTRACT prints -dE/d(euler), -dE/dt
    assert np.all(np.abs(E - refE) <= 2e-4 * np.abs(refE) + 2e-3), np.abs(E - refE).max()
    err = np.linalg.norm(-grad - refG, axis=1) / np.linalg.norm(refG, axis=1)
    assert err.max() < 1e-4, err.max()


# Pose 6 of the JAX runs lost pair terms to the coverage of ATTRACT's own
# nbgrid file (absent from the reference); the complete-list restatement
# cannot reproduce that, so it is excluded.  The JAX runs are float32, so the
# tolerances are float32 summation error over ~1e3 pair terms.
JAX_POSES = [0, 1, 2, 3, 4, 5, 7, 8, 9]


def _check_jax(E, dM, golden, key):
    i = JAX_POSES
    refE = golden[key + "_energy"][i]
    assert np.all(np.abs(E[i] - refE) <= 2e-5 * np.abs(refE) + 2e-3)
    assert np.all(np.abs(-dM[i, 3, :3] - golden[key + "_negdt"][i]) <= 1e-4 * np.abs(golden[key + "_negdt"][i]) + 3e-3)
    refM = golden[key + "_negdM"][i]
    scale = np.abs(refM).max((1, 2))[:, None, None]
    assert np.all(np.abs(-dM[i, :3, :3] - refM) <= 1e-5 * scale)


def test_nb_plain_vs_jax_out(golden, nb_plain):
    lig, gt, lt = _lig(golden)
    E, dM = O.energrad_mat(golden["mat10"], lig, gt, lt, nb_plain)
    _check_jax(E, dM, golden, "jax_nb")


def test_nb_plateau_vs_jax_out(golden, nb_plat):
    """test5 semantics: E(d)-E(plateau) and the custom-JVP gradient."""
    lig, gt, lt = _lig(golden)
    E, dM = O.energrad_mat(golden["mat10"], lig, gt, lt, nb_plat)
    _check_jax(E, dM, golden, "jax_nbplat")


def test_euler_gradient_consistent_with_mat_gradient(golden, nb_plat):
    pose = dat_poses(golden)[:4]
    lig, gt, lt = _lig(golden)
    E1, g = O.energrad(pose, lig, gt, lt, nb_plat)
    E2, dM = O.energrad_mat(O.pose_to_mat(pose), lig, gt, lt, nb_plat)
    assert np.allclose(E1, E2)
    assert np.allclose(g[:, 3:], dM[:, 3, :3])
    # rotational part by the chain rule through the matrix entries
    h = 1e-6
    for k in range(3):
        pp, pm = pose.copy(), pose.copy()
        pp[:, k] += h
        pm[:, k] -= h
        dmat = (O.pose_to_mat(pp) - O.pose_to_mat(pm)) / (2 * h)
        chain = (dmat[:, :3, :3] * dM[:, :3, :3]).sum((1, 2))
        assert np.allclose(chain, g[:, k], rtol=1e-6, atol=1e-4)


@settings(max_examples=25, deadline=None)
@given(seed=st.integers(0, 10_000), shift=st.tuples(*[st.floats(-20.0, 20.0)] * 3))
def test_oracle_energy_is_translation_invariant(seed, shift):
    """Moving the receptor, the grid origin and every pose by the same vector
    leaves the oracle's energies and pose gradients unchanged (FP64): the
    grid, list and pair terms depend only on relative positions."""
    from gpu_cases import small_case

    c = small_case(seed=seed, n_poses=12)
    G = c["G"]
    v = np.asarray(shift)
    G2 = dict(G)
    G2["geom"] = dict(G["geom"], origin=np.asarray(G["geom"]["origin"]) + v)
    G2["rec"] = G["rec"] + v
    poses2 = c["poses"].copy()
    poses2[:, 3:] += v
    E1, g1 = O.energrad(c["poses"], c["lig"], c["gt"], c["lt"], G)
    E2, g2 = O.energrad(poses2, c["lig"], c["gt"], c["lt"], G2)
    scale = np.abs(E1) + 1.0
    assert np.all(np.abs(E1 - E2) <= 1e-9 * scale)
    assert np.allclose(g1, g2, rtol=1e-7, atol=1e-7 * scale.max())
