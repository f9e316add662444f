"""Host side of the scoring / minimisation path: workloads, launches, graphs.

A :class:`Workload` is what one launch serves: up to 8 resident grids, a
:class:`LigandSet`, and *segments* -- runs of consecutive poses that share a
grid and a ligand (the reference scores one receptor and one ligand or
conformer ensemble per call, test5.py:411; a segment generalises that to many
in one launch).  Poses live in one ``[B, 6]`` float32 tensor in segment order.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import NamedTuple, Sequence

import numpy as np
import torch

from . import _lib
from .grid import Grid, _dev
from .ligand import LigandSet


@dataclass
class EvalOptions:
    grad_mode: str = "reference"   # "reference" (test5.py:310 forces) or "analytic"
    quirk: bool = True             # reference floor/ceil trilinear weights (test5.py:256-259)
    gravity: float = 0.0           # + gravity*|t|^2 (test5.py:419 uses 0.1)

    def to_c(self, pose_format: int = 0) -> _lib.AttEvalCfg:
        if self.grad_mode not in ("reference", "analytic"):
            raise ValueError(f"grad_mode {self.grad_mode!r}")
        c = _lib.AttEvalCfg()
        c.grad_mode = _lib.ATT_GRAD_REFERENCE if self.grad_mode == "reference" else _lib.ATT_GRAD_ANALYTIC
        c.flags = _lib.ATT_FLAG_TRILINEAR_QUIRK if self.quirk else 0
        c.gravity = float(self.gravity)
        c.pose_format = pose_format
        return c


@dataclass
class AdamOptions:
    lr_rot: float = 0.01    # rad
    lr_trans: float = 0.05  # Angstrom
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    step0: int = 0

    def to_c(self, ev: EvalOptions) -> _lib.AttAdamCfg:
        c = _lib.AttAdamCfg()
        c.eval = ev.to_c(0)
        c.lr_rot, c.lr_trans = float(self.lr_rot), float(self.lr_trans)
        c.beta1, c.beta2, c.eps = float(self.beta1), float(self.beta2), float(self.eps)
        c.step0 = int(self.step0)
        return c


@dataclass
class LaunchShape:
    lanes_per_pose: int = 8   # 8 / 16 / 32 lanes per pose = 4 / 2 / 1 poses per warp
    block_threads: int = 0    # 32, 64, 96 or 128; 0 = the largest that fits in shared memory
    blocks: int = 0           # persistent CTAs; 0 = fill the GPU
    test_flags: int = 0       # reserved: 0

    def to_c(self) -> _lib.AttLaunchCfg:
        c = _lib.AttLaunchCfg()
        c.lanes_per_pose, c.block_threads, c.blocks = self.lanes_per_pose, self.block_threads, self.blocks
        c.test_flags = self.test_flags
        return c

    @property
    def poses_per_warp(self) -> int:
        return 32 // self.lanes_per_pose


class Segment(NamedTuple):
    grid: int
    lig: int
    n_poses: int
    step0: int = 0            # ADAM steps already taken by these poses' state
    pose0: int | None = None  # first pose in the pose array (None: packed in segment order)


def _stream(stream):
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


def _used_on(stream, *tensors):
    """A launch on ``stream`` (not the current stream) reads or writes
    ``tensors``, which the caching allocator assigned to the current stream:
    record the use, so that their memory is not handed out again before that
    stream's work is done."""
    if stream is None:
        return
    s = stream if isinstance(stream, torch.cuda.Stream) else torch.cuda.ExternalStream(int(stream))
    if s.cuda_stream == torch.cuda.current_stream().cuda_stream:
        return
    for t in tensors:
        if t is not None:
            t.record_stream(s)


class Workload:
    """Device tables for launches over ``segments`` (see module docstring)."""

    def __init__(self, grids: Sequence[Grid], ligands: LigandSet, segments: Sequence[Segment],
                 lanes_per_pose: int = 8, device=None, n_poses: int | None = None):
        """``n_poses``: size of the pose array when segments give explicit
        ``pose0`` offsets (a pose pool); otherwise segments are packed in order."""
        if not 1 <= len(grids) <= _lib.ATT_MAX_GRIDS:
            raise ValueError(f"1..{_lib.ATT_MAX_GRIDS} grids per launch, got {len(grids)}")
        if lanes_per_pose not in (8, 16, 32):
            raise ValueError("lanes_per_pose must be 8, 16 or 32")
        self.device = _dev(device if device is not None else grids[0].device)
        self.grids = list(grids)
        self.ligands = ligands
        self.segments = [Segment(*s) for s in segments]
        if not self.segments:
            raise ValueError("no segments")
        explicit = [s.pose0 is not None for s in self.segments]
        if any(explicit) and not (all(explicit) and n_poses is not None):
            raise ValueError("explicit pose0 needs pose0 on every segment and n_poses")
        self.lanes = lanes_per_pose
        P = 32 // lanes_per_pose
        rows, tiles, pose0 = [], [0], 0
        for s in self.segments:
            if s.pose0 is not None:
                if s.pose0 < 0 or s.pose0 + s.n_poses > n_poses:
                    raise ValueError(f"segment {s} lies outside the {n_poses}-pose array")
                pose0 = s.pose0
            if s.step0 < 0:
                raise ValueError("negative step0")
            if not (0 <= s.grid < len(grids)) or not (0 <= s.lig < len(ligands)):
                raise ValueError(f"segment {s} refers to a missing grid or ligand")
            if s.n_poses < 0:
                raise ValueError("negative pose count")
            g = grids[s.grid]
            _, gt, lt = ligands.host[s.lig]
            if g.bricks is not None and gt.max() >= g.geom.n_types:
                raise ValueError(f"ligand {s.lig}: grid type {gt.max()} >= grid {s.grid}'s {g.geom.n_types} slots")
            if lt.max() >= g.ff.n_ltypes:
                raise ValueError(f"ligand {s.lig}: ligand type {lt.max()} outside grid {s.grid}'s force field")
            rows.append((s.grid, s.lig, pose0, s.n_poses, s.step0, 0, 0, 0))
            tiles.append(tiles[-1] + (s.n_poses + P - 1) // P)
            pose0 += s.n_poses
        self.n_poses = pose0 if n_poses is None else int(n_poses)
        self._pool = n_poses is not None
        self.n_tiles = tiles[-1]
        self.pose0 = [r[2] for r in rows]
        self.segs = torch.tensor(rows, dtype=torch.int32, device=self.device)
        self.seg_tile = torch.tensor(tiles, dtype=torch.int32, device=self.device)
        self.c_grids = (_lib.AttGrid * len(grids))(*[g.att() for g in grids])
        self.c_ligs = ligands.att()
        self.bead_counts = np.array([ligands.sizes[s.lig] for s in self.segments])

    def with_lanes(self, lanes_per_pose: int) -> "Workload":
        if lanes_per_pose == self.lanes:
            return self
        return Workload(self.grids, self.ligands, self.segments, lanes_per_pose, self.device,
                        self.n_poses if self._pool else None)

    def bead_evals(self, evals_per_pose: int) -> int:
        return int(sum(self.ligands.sizes[s.lig] * s.n_poses for s in self.segments)) * evals_per_pose

    def check_poses(self, poses: torch.Tensor, width: int = 6):
        if poses.device != self.device or poses.dtype != torch.float32 or not poses.is_contiguous():
            raise ValueError("poses must be a contiguous float32 tensor on the workload's device")
        if poses.shape != (self.n_poses, width):
            raise ValueError(f"poses shape {tuple(poses.shape)} != {(self.n_poses, width)}")


def energrad(wl: Workload, poses: torch.Tensor, opts: EvalOptions | None = None, *, grad: bool = True,
             pose_lig: torch.Tensor | None = None, launch: LaunchShape | None = None, stream=None,
             out=None):
    """One evaluation of every pose: ``(E [B], dE/dpose [B,6] or None, status [B])``.

    ``poses`` is ``[B, 6]`` Euler+translation or ``[B, 4, 4]`` / ``[B, 16]``
    row-vector matrices (then the gradient is dE/dmat ``[B, 4, 4]``).
    """
    opts = opts or EvalOptions()
    launch = launch or LaunchShape(lanes_per_pose=wl.lanes)
    if launch.lanes_per_pose != wl.lanes:
        raise ValueError("launch.lanes_per_pose differs from the workload's tiling")
    mat = poses.dim() == 3 or (poses.dim() == 2 and poses.shape[1] == 16)
    p2 = poses.reshape(len(poses), 16) if mat else poses
    wl.check_poses(p2, 16 if mat else 6)
    B = wl.n_poses
    if out is None:
        E = torch.empty(B, dtype=torch.float32, device=wl.device)
        G = torch.empty((B, 16 if mat else 6), dtype=torch.float32, device=wl.device) if grad else None
        S = torch.empty(B, dtype=torch.int32, device=wl.device)
    else:
        E, G, S = out
    if pose_lig is not None:
        _check_pose_lig(wl, pose_lig)
    cfg = opts.to_c(1 if mat else 0)
    lc = launch.to_c()
    rc = _lib.load().att_energrad(wl.c_grids, len(wl.grids), C.byref(wl.c_ligs), _lib.ptr(wl.segs),
                                  len(wl.segments), _lib.ptr(wl.seg_tile), wl.n_tiles, wl.n_poses, _lib.ptr(p2),
                                  _lib.ptr(pose_lig), C.byref(cfg), _lib.ptr(E), _lib.ptr(G), _lib.ptr(S),
                                  C.byref(lc), _stream(stream))
    _lib.check(rc, "att_energrad")
    _used_on(stream, wl.segs, wl.seg_tile, p2, pose_lig, E, G, S)
    if G is not None and mat:
        G = G.view(B, 4, 4)
    return E, G, S


def _check_pose_lig(wl: Workload, pose_lig: torch.Tensor):
    if pose_lig.dtype != torch.int32 or pose_lig.device != wl.device or pose_lig.shape != (wl.n_poses,):
        raise ValueError("pose_lig must be an int32 [B] tensor on the workload's device")
    sizes = np.array(wl.ligands.sizes)
    pl = pose_lig.cpu().numpy()
    for s, p0 in zip(wl.segments, wl.pose0):
        idx = s.lig + pl[p0:p0 + s.n_poses]
        if len(idx) and (idx.min() < 0 or idx.max() >= len(sizes)):
            raise ValueError("pose_lig points outside the ligand set")
        if len(idx) and np.any(sizes[idx] != sizes[s.lig]):
            raise ValueError("conformers of one segment must have equal bead counts")


def minimise(wl: Workload, poses: torch.Tensor, steps: int, adam: AdamOptions | None = None,
             opts: EvalOptions | None = None, *, pose_out: torch.Tensor | None = None,
             adam_state: torch.Tensor | None = None, pose_lig: torch.Tensor | None = None,
             launch: LaunchShape | None = None, stats: bool = False, stream=None, scratch=None):
    """Fused ADAM minimisation; returns ``(pose_out, E_final, status, stats)``."""
    adam = adam or AdamOptions()
    opts = opts or EvalOptions()
    launch = launch or LaunchShape(lanes_per_pose=wl.lanes)
    if launch.lanes_per_pose != wl.lanes:
        raise ValueError("launch.lanes_per_pose differs from the workload's tiling")
    wl.check_poses(poses)
    B = wl.n_poses
    if pose_out is None:
        pose_out = torch.empty_like(poses)
    if adam_state is not None and (adam_state.shape != (B, 12) or adam_state.dtype != torch.float32):
        raise ValueError("adam_state must be float32 [B, 12]")
    if pose_lig is not None:
        _check_pose_lig(wl, pose_lig)
    if scratch is None:
        scratch = MinimiseScratch(B, wl.device)
    st = torch.zeros(5, dtype=torch.int64, device=wl.device) if stats else None
    cfg = adam.to_c(opts)
    lc = launch.to_c()
    rc = _lib.load().att_minimise(wl.c_grids, len(wl.grids), C.byref(wl.c_ligs), _lib.ptr(wl.segs),
                                  len(wl.segments), _lib.ptr(wl.seg_tile), wl.n_tiles, wl.n_poses, _lib.ptr(poses),
                                  _lib.ptr(pose_out), _lib.ptr(pose_lig), _lib.ptr(adam_state), C.byref(cfg),
                                  int(steps), _lib.ptr(scratch.energy), _lib.ptr(scratch.status),
                                  _lib.ptr(scratch.counter), _lib.ptr(st), C.byref(lc), _stream(stream))
    _lib.check(rc, "att_minimise")
    _used_on(stream, wl.segs, wl.seg_tile, poses, pose_out, pose_lig, adam_state, scratch.energy, scratch.status,
             scratch.counter, st)
    return pose_out, scratch.energy, scratch.status, st


def minimise_schema(wl: Workload, poses: torch.Tensor, schema, opts: EvalOptions | None = None, *,
                    gravity_weight: float = 0.1, betas=(0.9, 0.999), eps: float = 1e-16, eps_root: float = 1e-16,
                    pose_out: torch.Tensor | None = None, pose_lig: torch.Tensor | None = None,
                    launch: LaunchShape | None = None, stream=None, scratch=None):
    """The reference's SCHEMA protocol (quaternion poses, optax.adabelief per
    stage, gravity per stage) in one persistent launch: ``poses`` is ``[B, 8]``
    (qx, qy, qz, qw, tx, ty, tz, unused); ``schema`` a sequence of (epochs,
    learning rate, gravity on) stages.  Returns ``(pose_out [B, 8], E of the
    last evaluation [B], status [B])``."""
    opts = opts or EvalOptions()
    launch = launch or LaunchShape(lanes_per_pose=wl.lanes)
    if launch.lanes_per_pose != wl.lanes:
        raise ValueError("launch.lanes_per_pose differs from the workload's tiling")
    wl.check_poses(poses, 8)
    stages = [tuple(st) for st in schema]
    if not 1 <= len(stages) <= _lib.ATT_MAX_STAGES:
        raise ValueError(f"1..{_lib.ATT_MAX_STAGES} schema stages")
    if pose_out is None:
        pose_out = torch.empty_like(poses)
    if pose_lig is not None:
        _check_pose_lig(wl, pose_lig)
    if scratch is None:
        scratch = MinimiseScratch(wl.n_poses, wl.device)
    cfg = _lib.AttSchemaCfg()
    cfg.eval = EvalOptions(opts.grad_mode, opts.quirk, gravity_weight).to_c(0)
    cfg.n_stages = len(stages)
    for i, (ep, lr, grav) in enumerate(stages):
        cfg.epochs[i], cfg.lr[i], cfg.gravity[i] = int(ep), float(lr), int(bool(grav))
    cfg.beta1, cfg.beta2, cfg.eps, cfg.eps_root = float(betas[0]), float(betas[1]), float(eps), float(eps_root)
    lc = launch.to_c()
    rc = _lib.load().att_minimise_schema(wl.c_grids, len(wl.grids), C.byref(wl.c_ligs), _lib.ptr(wl.segs),
                                         len(wl.segments), _lib.ptr(wl.seg_tile), wl.n_tiles, wl.n_poses, _lib.ptr(poses),
                                         _lib.ptr(pose_out), _lib.ptr(pose_lig), C.byref(cfg),
                                         _lib.ptr(scratch.energy), _lib.ptr(scratch.status),
                                         _lib.ptr(scratch.counter), C.byref(lc), _stream(stream))
    _lib.check(rc, "att_minimise_schema")
    _used_on(stream, wl.segs, wl.seg_tile, poses, pose_out, pose_lig, scratch.energy, scratch.status, scratch.counter)
    return pose_out, scratch.energy, scratch.status


class MinimiseScratch:
    """Output and work-queue buffers of one minimisation launch."""

    def __init__(self, n_poses: int, device):
        self.energy = torch.empty(max(n_poses, 1), dtype=torch.float32, device=device)[:n_poses]
        self.status = torch.empty(max(n_poses, 1), dtype=torch.int32, device=device)[:n_poses]
        self.counter = torch.zeros(1, dtype=torch.int32, device=device)


def energrad_backward(wl: Workload, poses: torch.Tensor, dL_dE: torch.Tensor, opts: EvalOptions | None = None,
                      dgrid_inner: torch.Tensor | None = None, dgrid_outer: torch.Tensor | None = None,
                      pose_lig: torch.Tensor | None = None, launch: LaunchShape | None = None, stream=None):
    """Adjoint of :func:`energrad`: returns dL/dpose and scatter-adds dL/d(grid energies)."""
    opts = opts or EvalOptions()
    launch = launch or LaunchShape(lanes_per_pose=wl.lanes)
    wl.check_poses(poses)
    dL_dE = dL_dE.contiguous().to(torch.float32)
    if dL_dE.shape != (wl.n_poses,):
        raise ValueError("dL_dE must be [B]")
    out = torch.empty_like(poses)
    cfg = opts.to_c(0)
    lc = launch.to_c()
    rc = _lib.load().att_energrad_backward(wl.c_grids, len(wl.grids), C.byref(wl.c_ligs), _lib.ptr(wl.segs),
                                           len(wl.segments), _lib.ptr(wl.seg_tile), wl.n_tiles, wl.n_poses, _lib.ptr(poses),
                                           _lib.ptr(pose_lig), C.byref(cfg), _lib.ptr(dL_dE), _lib.ptr(out),
                                           _lib.ptr(dgrid_inner), _lib.ptr(dgrid_outer), C.byref(lc),
                                           _stream(stream))
    _lib.check(rc, "att_energrad_backward")
    _used_on(stream, wl.segs, wl.seg_tile, poses, pose_lig, dL_dE, out, dgrid_inner, dgrid_outer)
    return out


class MinimisePlan:
    """A fixed minimisation launch (buffers bound once) that can be captured
    into a CUDA graph and replayed: the batched path launches all segments --
    many ligands of uneven bead and pose counts -- as one persistent kernel."""

    def __init__(self, wl: Workload, steps: int, adam: AdamOptions | None = None, opts: EvalOptions | None = None,
                 launch: LaunchShape | None = None, pose_lig: torch.Tensor | None = None):
        self.wl = wl
        self.steps = steps
        self.adam = adam or AdamOptions()
        self.opts = opts or EvalOptions()
        self.launch = launch or LaunchShape(lanes_per_pose=wl.lanes)
        self.pose_in = torch.zeros((wl.n_poses, 6), dtype=torch.float32, device=wl.device)
        self.pose_out = torch.zeros_like(self.pose_in)
        self.pose_lig = pose_lig
        self.scratch = MinimiseScratch(wl.n_poses, wl.device)
        self.graph = None

    def run(self, stream=None):
        return minimise(self.wl, self.pose_in, self.steps, self.adam, self.opts, pose_out=self.pose_out,
                        pose_lig=self.pose_lig, launch=self.launch, stream=stream, scratch=self.scratch)

    def capture(self):
        s = torch.cuda.Stream(self.wl.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.run()  # warm (loads the library, validates arguments)
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()
        return self.pose_out, self.scratch.energy, self.scratch.status
