"""Pose conventions.

A pose is ``(phi, psi, theta, tx, ty, tz)`` in ATTRACT ``.dat`` order.  The
reference's row-vector matrix (test5.py:413-415) is
``mat[:3,:3] = Rz(theta) Ry(-psi) Rz(-phi)`` -- scipy
``Rotation.from_euler('zyz', [-phi, -psi, theta])`` -- and ``mat[3,:3] = t``;
a bead moves to ``[x, 1] @ mat``.  The column form of the rotation is
``Q = Rz(phi) Ry(psi) Rz(-theta)``.
"""
from __future__ import annotations

import numpy as np


def euler_to_Q(phi, psi, theta) -> np.ndarray:
    cp, sp = np.cos(phi), np.sin(phi)
    cs, ss = np.cos(psi), np.sin(psi)
    ct, st = np.cos(theta), np.sin(theta)
    Q = np.empty(np.shape(phi) + (3, 3))
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


def Q_to_euler(Q) -> np.ndarray:
    """(phi, psi, theta) of a proper rotation in the convention above."""
    Q = np.asarray(Q, np.float64)
    psi = np.arccos(np.clip(Q[..., 2, 2], -1.0, 1.0))
    phi = np.arctan2(Q[..., 1, 2], Q[..., 0, 2])
    theta = np.arctan2(-Q[..., 2, 1], -Q[..., 2, 0])
    return np.stack([phi, psi, theta], -1)


def pose_to_mat(pose) -> np.ndarray:
    pose = np.asarray(pose, np.float64)
    mat = np.ones(pose.shape[:-1] + (4, 4))
    mat[..., :3, :3] = np.swapaxes(euler_to_Q(pose[..., 0], pose[..., 1], pose[..., 2]), -1, -2)
    mat[..., 3, :3] = pose[..., 3:6]
    return mat


def mat_to_pose(mat) -> np.ndarray:
    mat = np.asarray(mat, np.float64)
    ang = Q_to_euler(np.swapaxes(mat[..., :3, :3], -1, -2))
    return np.concatenate([ang, mat[..., 3, :3]], -1)


def quat_to_Q(q) -> np.ndarray:
    """Scalar-last unit quaternion (x, y, z, w) -> column rotation matrix."""
    q = np.asarray(q, np.float64)
    q = q / np.linalg.norm(q, axis=-1, keepdims=True)
    x, y, z, w = np.moveaxis(q, -1, 0)
    Q = np.empty(q.shape[:-1] + (3, 3))
    Q[..., 0, 0] = 1 - 2 * (y * y + z * z)
    Q[..., 0, 1] = 2 * (x * y - z * w)
    Q[..., 0, 2] = 2 * (x * z + y * w)
    Q[..., 1, 0] = 2 * (x * y + z * w)
    Q[..., 1, 1] = 1 - 2 * (x * x + z * z)
    Q[..., 1, 2] = 2 * (y * z - x * w)
    Q[..., 2, 0] = 2 * (x * z - y * w)
    Q[..., 2, 1] = 2 * (y * z + x * w)
    Q[..., 2, 2] = 1 - 2 * (x * x + y * y)
    return Q


def random_rotations(n: int, rng) -> np.ndarray:
    """Uniform rotations on SO(3) (Shoemake's subgroup algorithm), as Euler angles."""
    u1, u2, u3 = rng.random((3, n))
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], -1)
    return Q_to_euler(quat_to_Q(q))


def random_in_ball(n: int, radius: float, rng, centre=(0.0, 0.0, 0.0)) -> np.ndarray:
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * rng.random(n) ** (1.0 / 3.0)
    return np.asarray(centre) + d * r[:, None]
