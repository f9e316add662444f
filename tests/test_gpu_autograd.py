"""The adjoint kernel behind torch.autograd (differentiation workload).

* dL/d(pose), analytic gradient mode, against float64 central finite
  differences (h = 1e-4) of the oracle energy;
* dL/d(grid energy value) at sampled voxels against float64 central finite
  differences of the oracle's summed energy (linear in the grid values, so
  the finite difference is exact up to rounding);
* reference gradient mode: the backward pose gradient is dL/dE times the
  forward kernel's gradient.
"""
import numpy as np
import pytest
import torch

import attract_oracle as O
from gpu_cases import small_case, to_device_grid

pytestmark = pytest.mark.gpu


def _setup(seed=30, n_poses=64):
    import attract_b200 as A
    from attract_b200.autograd import docking_energy

    A.load_library()
    c = small_case(seed=seed, n_poses=n_poses)
    grid = to_device_grid(c)
    wl = A.Workload([grid], A.LigandSet([(c["lig"], c["gt"], c["lt"])]), [A.Segment(0, 0, n_poses)])
    return A, docking_energy, c, grid, wl


def test_pose_gradient_vs_fp64_finite_differences():
    A, docking_energy, c, grid, wl = _setup()
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda", requires_grad=True)
    E = docking_energy(wl, P, A.EvalOptions(grad_mode="analytic"))
    E.backward()
    g = P.grad.cpu().numpy().astype(np.float64)
    h = 1e-4
    fd = np.zeros_like(g)
    for k in range(6):
        pp, pm = c["poses"].copy(), c["poses"].copy()
        pp[:, k] += h
        pm[:, k] -= h
        Ep, _ = O.energrad(pp, c["lig"], c["gt"], c["lt"], c["G"], mode="analytic")
        Em, _ = O.energrad(pm, c["lig"], c["gt"], c["lt"], c["G"], mode="analytic")
        fd[:, k] = (Ep - Em) / (2 * h)
    _, ga = O.energrad(c["poses"], c["lig"], c["gt"], c["lt"], c["G"], mode="analytic")
    scale = np.abs(ga).max(1, keepdims=True) + 1.0
    # the kernel matches the float64 analytic gradient everywhere ...
    assert np.all(np.abs(g - ga) <= 2e-4 * scale), np.abs(g - ga).max()
    # ... and finite differences wherever no bead crosses a voxel face or the plateau within +-h
    ok = np.all(np.abs(fd - ga) <= 1e-3 * scale, axis=1)
    assert ok.mean() > 0.9, ok.mean()
    assert np.all(np.abs(g - fd)[ok] <= 2e-3 * scale[ok])


def test_grid_gradient_vs_fp64_finite_differences():
    A, docking_energy, c, grid, wl = _setup(seed=31)
    grid.inner.requires_grad_(True)
    grid.outer.requires_grad_(True)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    E = docking_energy(wl, P, A.EvalOptions(grad_mode="analytic"))
    E.backward()
    din = grid.inner.grad.cpu().numpy()
    dout = grid.outer.grad.cpu().numpy()
    assert np.all(din[..., 1:] == 0) and np.all(dout[..., 1:] == 0)
    rng = np.random.default_rng(0)
    touched = np.argwhere(din[..., 0] != 0)
    pick = touched[rng.choice(len(touched), min(128, len(touched)), replace=False)]
    pick = np.concatenate([pick, np.stack([rng.integers(0, n, 64) for n in din.shape[:4]], 1)])
    touched_o = np.argwhere(dout[..., 0] != 0)
    h = 1e-4
    G = dict(c["G"])
    for which, arr, pts in (("inner", din, pick), ("outer", dout, touched_o[:64])):
        base = G[which].copy()
        for v in pts:
            t, x, y, z = (int(q) for q in v)
            gp, gm = base.copy(), base.copy()
            gp[t, x, y, z, 0] += h
            gm[t, x, y, z, 0] -= h
            Ep, _ = O.energrad(c["poses"], c["lig"], c["gt"], c["lt"], {**G, which: gp}, mode="analytic")
            Em, _ = O.energrad(c["poses"], c["lig"], c["gt"], c["lt"], {**G, which: gm}, mode="analytic")
            fd = (Ep.sum() - Em.sum()) / (2 * h)
            assert abs(arr[t, x, y, z, 0] - fd) <= 1e-5 * max(1.0, abs(fd)), (which, v, arr[t, x, y, z, 0], fd)


def test_reference_mode_backward_is_dLdE_times_forward_gradient():
    A, docking_energy, c, grid, wl = _setup(seed=32)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda", requires_grad=True)
    w = torch.linspace(-1.0, 2.0, len(c["poses"]), device="cuda")
    E = docking_energy(wl, P, A.EvalOptions(), reduce="none")
    (E * w).sum().backward()
    _, G, _ = A.energrad(wl, P.detach())
    assert torch.allclose(P.grad, w[:, None] * G, rtol=1e-5, atol=1e-4)


def test_grid_edit_is_repacked():
    """Changing the dense grid in place changes the next forward pass."""
    A, docking_energy, c, grid, wl = _setup(seed=33)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    E0 = docking_energy(wl, P, reduce="none").detach().clone()
    with torch.no_grad():
        grid.inner[..., 0] += 1.0
    E1 = docking_energy(wl, P, reduce="none").detach()
    G = dict(c["G"])
    G["inner"] = c["G"]["inner"].copy()
    G["inner"][..., 0] += 1.0
    Eo, _ = O.energrad(c["poses"], c["lig"], c["gt"], c["lt"], G)
    assert not torch.equal(E0, E1)
    assert np.allclose(E1.cpu().numpy(), Eo, rtol=1e-4, atol=1e-3)


def _host_scatter(c, poses, dLdE):
    """dL/d(grid energy value): the float64 host sum of dL/dE * trilinear weight
    over every bead and corner (inner grid where in range, else outer)."""
    G = c["G"]
    g = G["geom"]
    X = O.transform(poses, c["lig"])
    inner = np.zeros(G["inner"].shape[:4])
    outer = np.zeros(G["outer"].shape[:4])
    v = (X - np.asarray(g["origin"])) / g["spacing"]
    u = (v + g["extension"]) / 2.0
    dim, dim2 = np.asarray(g["dim"]), np.asarray(g["dim2"])
    for b in range(len(poses)):
        for i in range(len(c["lig"])):
            if np.all((v[b, i] >= 0) & (v[b, i] < dim - 1)):
                tgt, q = inner, v[b, i]
            elif np.all((u[b, i] >= 0) & (u[b, i] < dim2 - 1)):
                tgt, q = outer, u[b, i]
            else:
                continue
            base = np.floor(q).astype(int)
            f = q - base
            for cx in (0, 1):
                for cy in (0, 1):
                    for cz in (0, 1):
                        w = (f[0] if cx else 1 - f[0]) * (f[1] if cy else 1 - f[1]) * (f[2] if cz else 1 - f[2])
                        tgt[c["gt"][i], base[0] + cx, base[1] + cy, base[2] + cz] += dLdE[b] * w
    return inner, outer


def test_grid_scatter_equals_a_deterministic_host_sum():
    """The adjoint's atomic scatter into the dense grid gradient (every voxel)
    equals the float64 host sum up to float32 accumulation error; two runs
    agree to the same bound (atomics add in a varying order); the forward
    kernel is bitwise deterministic."""
    A, _, c, grid, wl = _setup(seed=34, n_poses=48)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    dLdE = torch.linspace(-1.0, 2.0, 48, device="cuda")
    res = []
    for _ in range(2):
        di = torch.zeros((*grid.inner.shape[:4], 4), dtype=torch.float32, device="cuda")
        do = torch.zeros((*grid.outer.shape[:4], 4), dtype=torch.float32, device="cuda")
        A.energrad_backward(wl, P, dLdE, A.EvalOptions(grad_mode="analytic"), dgrid_inner=di, dgrid_outer=do)
        res.append((di[..., 0].cpu().numpy(), do[..., 0].cpu().numpy()))
        assert torch.all(di[..., 1:] == 0) and torch.all(do[..., 1:] == 0)
    hi, ho = _host_scatter(c, c["poses"].astype(np.float32).astype(np.float64), dLdE.cpu().numpy())
    scale = float(np.abs(dLdE.cpu().numpy()).sum())
    for got, ref in ((res[0][0], hi), (res[0][1], ho)):
        assert np.abs(got - ref).max() <= 1e-5 * scale, np.abs(got - ref).max()
    for a, b in zip(res[0], res[1]):
        assert np.abs(a - b).max() <= 1e-5 * scale
    E1, G1, _ = A.energrad(wl, P)
    E2, G2, _ = A.energrad(wl, P)
    assert torch.equal(E1, E2) and torch.equal(G1, G2)


def test_backward_refuses_bricks_repacked_after_its_forward():
    """The backward recomputes its forward from the bricks: if another forward
    repacked them from edited dense grids in between, it raises instead of
    returning gradients of the new grid."""
    A, docking_energy, c, grid, wl = _setup(seed=35)
    grid.inner.requires_grad_(True)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda", requires_grad=True)
    E0 = docking_energy(wl, P)
    with torch.no_grad():
        grid.inner[..., 0] += 0.5
    E1 = docking_energy(wl, P)  # repacks
    with pytest.raises(RuntimeError, match="repacked"):
        E0.backward()
    E1.backward()  # the latest forward still differentiates
    assert torch.isfinite(P.grad).all()
