"""Differentiable docking energy: a torch.autograd.Function over the kernels.

The reference differentiates its scorer with ``jax.value_and_grad`` with
respect to the pose (test5.py:429).  Here the forward pass is the fused
energy kernel and the backward pass is the hand-written adjoint kernel
(``att_energrad_backward``), which recomputes the forward per bead instead of
storing corner weights, and returns both

* dL/d(pose) ``[B, 6]`` = dL/dE * dE/d(phi, psi, theta, t), and
* dL/d(grid energy values): scatter-added into tensors shaped like the dense
  inner / outer grids ``[T, dx, dy, dz, 4]`` (channel 0; the force channels
  do not enter the energy).

``grad_mode='analytic'`` makes dE/d(pose) the exact derivative of the
computed energy (finite-difference consistent); ``'reference'`` is the
reference's gradient (interpolated stored forces, plateau-corrected pairs).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .engine import EvalOptions, Workload, energrad, energrad_backward


class DockingEnergy(torch.autograd.Function):
    """E[b] for every pose; differentiable in ``poses`` and in the grid's dense
    inner/outer energy grids (which must be the tensors the grid's bricks are
    packed from: ``Grid.build(..., keep_dense=True)`` / ``Grid.from_dense``)."""

    @staticmethod
    def forward(ctx, poses, inner, outer, wl: Workload, opts: EvalOptions):
        grid = wl.grids[0]
        _sync_bricks(grid, inner, outer)
        E, _, _ = energrad(wl, poses.detach().contiguous(), opts, grad=False)
        ctx.save_for_backward(poses)
        ctx.wl, ctx.opts = wl, opts
        ctx.packed_version = getattr(grid, "_packed_version", None)
        ctx.has_inner, ctx.has_outer = inner is not None, outer is not None
        return E

    @staticmethod
    def backward(ctx, dE):
        (poses,) = ctx.saved_tensors
        wl, opts = ctx.wl, ctx.opts
        grid = wl.grids[0]
        if getattr(grid, "_packed_version", None) != ctx.packed_version:
            # the backward recomputes the forward from the bricks: another
            # forward repacked them from modified dense grids in between
            raise RuntimeError("the grid's bricks were repacked from modified dense grids after this forward; "
                               "its backward would use the new grid values")
        need_grid = ctx.needs_input_grad[1] or ctx.needs_input_grad[2]
        din = torch.zeros_like(grid.inner) if (need_grid and ctx.has_inner) else None
        dout = torch.zeros_like(grid.outer) if (need_grid and ctx.has_outer) else None
        dpose = energrad_backward(wl, poses.detach().contiguous(), dE.detach().contiguous(), opts, din, dout)
        return (dpose if ctx.needs_input_grad[0] else None), din, dout, None, None


def _sync_bricks(grid, inner, outer):
    """Repack the bricks when the dense grids changed since they were packed."""
    if inner is None:
        return
    if inner is not grid.inner or (outer is not None and outer is not grid.outer):
        raise ValueError("pass the grid's own dense tensors (grid.inner / grid.outer)")
    ver = (inner._version, None if outer is None else outer._version)
    if getattr(grid, "_packed_version", None) == ver:
        return
    gc = grid.geom.to_c()
    st = torch.cuda.current_stream(grid.device).cuda_stream
    _lib.check(_lib.load().att_grid_repack(C.byref(gc), _lib.ptr(inner.detach()),
                                           _lib.ptr(None if outer is None else outer.detach()),
                                           _lib.ptr(grid.bricks), st), "att_grid_repack")
    grid._packed_version = ver


def docking_energy(wl: Workload, poses: torch.Tensor, opts: EvalOptions | None = None, reduce: str = "sum"):
    """Differentiable energies of ``poses`` on the workload's (single) grid.

    ``reduce='sum'`` returns the summed energy (a scalar), ``'none'`` the
    per-pose energies.  Gradients flow to ``poses`` and, when they require
    grad, to ``wl.grids[0].inner`` / ``.outer``.
    """
    if len(wl.grids) != 1:
        raise ValueError("docking_energy differentiates one grid at a time")
    grid = wl.grids[0]
    E = DockingEnergy.apply(poses, grid.inner, grid.outer, wl, opts or EvalOptions())
    return E.sum() if reduce == "sum" else E
