"""Host logic of the reference call surface (attract_b200.reference_api) on the
CPU: quaternion -> matrix and its chain rule, the adabelief update and the
argument checks, against the oracle's independent restatements."""
import numpy as np
import pytest
import torch

import attract_oracle as O
from attract_b200 import reference_api as R


def _quats(n, seed):
    q = np.random.default_rng(seed).normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def test_quat_matrix_matches_scipy_rotation():
    from scipy.spatial.transform import Rotation

    q = _quats(64, 0)
    ref = Rotation.from_quat(q).as_matrix()  # scalar-last, as jax.scipy's Rotation
    assert np.abs(O.quat_to_matrix(q) - ref).max() < 1e-14
    assert np.abs(R.quat_to_matrix(torch.tensor(q)).numpy() - ref).max() < 1e-14


def test_quat_chain_rule_matches_oracle_and_finite_differences():
    rng = np.random.default_rng(1)
    q = _quats(40, 2) * rng.uniform(0.5, 2.0, (40, 1))  # the form is homogeneous: any norm
    G = rng.normal(size=(40, 3, 3))
    ours = R.quat_grad(torch.tensor(q), torch.tensor(G)).numpy()
    assert np.abs(ours - O.quat_grad(q, G)).max() < 1e-12
    h = 1e-6
    fd = np.zeros_like(q)
    for i in range(4):
        d = np.zeros(4)
        d[i] = h
        fd[:, i] = ((O.quat_to_matrix(q + d) - O.quat_to_matrix(q - d)) * G).sum((1, 2)) / (2 * h)
    assert np.abs(ours - fd).max() < 1e-7


def test_adabelief_matches_oracle_update():
    rng = np.random.default_rng(3)
    p = [rng.normal(size=(10, 4)), rng.normal(size=(10, 3))]
    opt = R.AdaBelief([torch.tensor(x) for x in p], lr=0.5)
    mu = [np.zeros_like(x) for x in p]
    nu = [np.zeros_like(x) for x in p]
    for k in range(1, 6):
        g = [rng.normal(size=x.shape) for x in p]
        ours = opt.updates([torch.tensor(x) for x in g])
        for i in range(2):
            err = g[i] - mu[i]
            mu[i] = 0.9 * mu[i] + 0.1 * g[i]
            nu[i] = 0.999 * nu[i] + 0.001 * err * err + 1e-16
            ref = -0.5 * (mu[i] / (1 - 0.9 ** k)) / (np.sqrt(nu[i] / (1 - 0.999 ** k)) + 1e-16)
            assert np.allclose(ours[i].numpy(), ref, rtol=1e-12, atol=0)


def test_make_ff_follows_test5():
    rng = np.random.default_rng(4)
    rc, ac = rng.uniform(1e3, 1e5, (3, 2)), rng.uniform(10, 100, (3, 2))
    ff = R.make_ff(rc, ac, np.ones((3, 2)))
    assert np.allclose(ff.emin, -27.0 * ac ** 4 / (256.0 * rc ** 3))
    assert np.allclose(ff.rmin2, 4.0 * rc / (3.0 * ac))
    assert ff._fields == ("rc", "ac", "ivor", "emin", "rmin2")


def test_call_checks_follow_the_reference():
    q = _quats(5, 5)
    t = np.zeros((5, 3))
    assert R.check_call(q, t, np.arange(5))[0] == 5
    assert R.check_call(np.zeros((5, 3, 3)), t, None) == (5, None)
    with pytest.raises(AssertionError):
        R.check_call(q, np.zeros((4, 3)), None)  # test5.py:412
    with pytest.raises(AssertionError):
        R.check_call(q, t, np.arange(4))
    with pytest.raises(AssertionError):
        R.check_call(np.zeros((5, 3)), t, None)
    with pytest.raises(AssertionError):
        R.check_call(q, t, -np.ones(5))
