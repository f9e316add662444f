"""Continuous-batching docking server with receptor grids resident in HBM.

Requests (receptor, ligand, poses) are admitted while the pose pool and the
HBM budget allow, minimised in *rounds*: a round advances every admitted
request by ``round_steps`` ADAM steps, whatever its receptor, ligand size or
progress (each request is one segment of a launch with its own ADAM step
offset, its pose / ADAM state living in a slice of the pool).  The requests
of a round are grouped by *launch shape* -- lanes per pose and beads per lane,
both functions of the request's own ligand size -- and each group is one
persistent kernel launch, the groups on their own streams so that one
group's blocks fill the SMs another group's tail leaves idle.  (One launch for
all would size every pose's bead slots for the largest ligand present.)  A
request that arrives while others are on the GPU joins at the next round; a
finished request leaves and frees its slice.  The result of a request does
not depend on what it was batched with: per-pose arithmetic is independent
of the other poses of a launch, and the launch shape depends on the request
alone.

Rounds are pipelined: a round is enqueued while the previous one still runs
(at most ``max_rounds_in_flight``), so the GPU does not wait for the host's
admission and retirement work between rounds.  A request's last round copies
its results into a pinned host mirror of the pose pool on the same stream, and
the request is retired when that round's completion event has fired; its
pool rows are reused only by work enqueued after those copies.

Latency is wall-clock from ``submit`` to completion; ``stats()`` reports
p50/p99 latency and sustained poses/s.  Every finished request can be logged
as one JSON line (``log_path``), and :meth:`DockingServer.snapshot` /
:meth:`DockingServer.resume` checkpoint the unfinished ones between rounds:
a request's pose and ADAM state are per pose and tiny, so a resumed request
continues exactly where it stopped.  The phases of a round carry NVTX ranges.
"""
from __future__ import annotations

import bisect
import json
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from .engine import AdamOptions, EvalOptions, LaunchShape, Segment, Workload, minimise, MinimiseScratch
from .ligand import LigandSet

POSE_BYTES = 4 * (6 + 12 + 1 + 1)  # pose, ADAM state, energy, status


def _lig_copy(lig):
    return tuple(None if a is None else np.array(a) for a in lig)


@dataclass
class Request:
    receptor: int
    ligand: tuple            # (xyz [N,3], gtype [N], ltype [N] or None)
    poses: np.ndarray        # [n, 6]
    rid: int = -1
    arrival: float = 0.0
    admitted: float = 0.0
    finished: float = 0.0
    slot0: int = -1
    step: int = 0
    result_poses: np.ndarray | None = None
    result_energies: np.ndarray | None = None
    result_status: np.ndarray | None = None
    adam0: np.ndarray | None = None   # [n, 12] ADAM moments to start from (a resumed request)
    step0: int = 0                    # ADAM steps already taken (a resumed request)

    @property
    def n(self) -> int:
        return len(self.poses)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class PosePool:
    """First-fit allocator of contiguous pose ranges in [0, capacity)."""

    def __init__(self, capacity: int):
        self.capacity = capacity
        self.free = [(0, capacity)]  # sorted (start, length)

    def alloc(self, n: int) -> int:
        for i, (s, ln) in enumerate(self.free):
            if ln >= n:
                if ln == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (s + n, ln - n)
                return s
        return -1

    def release(self, s: int, n: int):
        """Return [s, s + n) to the pool; a range outside the pool or
        overlapping free space (a double release) raises ValueError."""
        if n <= 0 or s < 0 or s + n > self.capacity:
            raise ValueError(f"release of [{s}, {s + n}) outside the pool [0, {self.capacity})")
        i = bisect.bisect_left(self.free, (s, 0))
        if (i > 0 and self.free[i - 1][0] + self.free[i - 1][1] > s) or (i < len(self.free) and self.free[i][0] < s + n):
            raise ValueError(f"release of [{s}, {s + n}) overlaps free space (released twice?)")
        self.free.insert(i, (s, n))
        merged = []
        for a, ln in self.free:
            if merged and merged[-1][0] + merged[-1][1] == a:
                merged[-1] = (merged[-1][0], merged[-1][1] + ln)
            else:
                merged.append((a, ln))
        self.free = merged

    @property
    def used(self) -> int:
        return self.capacity - sum(ln for _, ln in self.free)


def lanes_by_size(n_beads: int) -> int:
    """Lanes per pose for a ligand: as many lanes as beads, rounded up to 8,
    16 or 32 (a smaller team puts more poses in a warp).  On the serving
    mix (ligands of 5-60 beads, four receptors) this policy beat 32 lanes
    for every request by 2.3 % and one launch for all shapes by 11 %."""
    return 8 if n_beads <= 8 else 16 if n_beads <= 16 else 32


def launch_order(r: "Request"):
    """Sort key of the requests within one launch: larger ligands first (their
    tiles take longest, so they do not end up in the launch's tail)."""
    return -len(r.ligand[0])


def launch_shape(n_beads: int, lanes: int) -> tuple[int, int]:
    """(lanes per pose, beads per lane) for a ligand of ``n_beads`` beads: the
    beads per lane the kernel picks for it (the next power of two of
    n_beads / lanes, at most 4; larger ligands run in chunks of 4)."""
    if lanes not in (8, 16, 32):
        raise ValueError(f"{lanes} lanes per pose: 8, 16 or 32")
    if n_beads < 1:
        raise ValueError("a ligand has at least one bead")
    k = 1
    while k < 4 and k * lanes < n_beads:
        k *= 2
    return lanes, k


class _GroupScratch:
    """The server's pool-wide energy / status buffers with one group's own
    work counter (groups that run concurrently need separate counters)."""

    def __init__(self, pool: MinimiseScratch, counter: torch.Tensor):
        self.energy, self.status, self.counter = pool.energy, pool.status, counter


class DockingServer:
    def __init__(self, grids, steps: int = 200, round_steps: int = 25, max_inflight_poses: int = 1_000_000,
                 hbm_budget_bytes: float = 150e9, adam: AdamOptions | None = None, opts: EvalOptions | None = None,
                 launch: LaunchShape | None = None, device=None, log_path: str | None = None,
                 lanes_for=None, concurrent: bool = True, max_rounds_in_flight: int = 2):
        """``launch``: block size / block count of every launch;
        ``lanes_for``: ligand bead count -> lanes per pose (8, 16 or 32),
        by default :func:`lanes_by_size`; ``concurrent``: the shape groups of
        a round run on their own streams (else one after another on the
        current stream); ``max_rounds_in_flight``: rounds enqueued on the GPU
        before the host waits for the oldest (1 = a synchronous loop)."""
        if steps % round_steps:
            raise ValueError("steps must be a multiple of round_steps")
        if len(grids) > 8:
            raise ValueError("at most 8 resident receptors per launch")
        self.grids = list(grids)
        self.device = self.grids[0].device if device is None else torch.device(device)
        self.steps, self.round_steps = steps, round_steps
        self.adam = adam or AdamOptions()
        self.opts = opts or EvalOptions()
        self.launch = launch or LaunchShape(lanes_per_pose=32)
        self.lanes_for = lanes_for or lanes_by_size
        self.concurrent = concurrent
        grid_bytes = sum(g.nbytes() for g in self.grids)
        cap = int(min(max_inflight_poses, max(0.0, hbm_budget_bytes - grid_bytes) // POSE_BYTES))
        if cap <= 0:
            raise ValueError("the HBM budget does not cover the resident grids")
        self.capacity = cap
        self.hbm_budget = hbm_budget_bytes
        self.grid_bytes = grid_bytes
        self.pool = PosePool(cap)
        d = self.device
        self.pose = torch.zeros((cap, 6), dtype=torch.float32, device=d)
        self.state = torch.zeros((cap, 12), dtype=torch.float32, device=d)
        self.scratch = MinimiseScratch(cap, d)
        # pinned host mirror of the pool's results (pose, energy, status), same rows
        self.h_pose = torch.empty((cap, 6), dtype=torch.float32).pin_memory()
        self.h_energy = torch.empty(cap, dtype=torch.float32).pin_memory()
        self.h_status = torch.empty(cap, dtype=torch.int32).pin_memory()
        self.max_rounds_in_flight = max(1, int(max_rounds_in_flight))
        self._inflight: deque = deque()  # (start event, end event, finishing requests, tables) per round
        self.pending: deque[Request] = deque()
        self.active: list[Request] = []
        self.done: list[Request] = []
        self._groups = {}   # launch shape -> (request ids, LigandSet, counter, stream)
        self.launches = 0
        self._next_rid = 0
        self.rounds = 0
        self.gpu_ms = 0.0
        self.t0 = time.perf_counter()
        self.log = open(log_path, "a") if log_path else None

    # ------------------------------------------------------------------ API
    def submit(self, req: Request, now: float | None = None) -> Request:
        if not 0 <= req.receptor < len(self.grids):
            raise ValueError("unknown receptor")
        if req.n > self.capacity:
            raise ValueError(f"request of {req.n} poses exceeds the pool of {self.capacity}")
        req.rid = self._next_rid
        self._next_rid += 1
        req.arrival = time.perf_counter() if now is None else now
        self.pending.append(req)
        return req

    def idle(self) -> bool:
        return not self.pending and not self.active and not self._inflight

    def run_until_idle(self):
        while not self.idle():
            self.round()
        self.drain()

    def drain(self):
        """Wait for every enqueued round and retire its finished requests."""
        while self._inflight:
            self._retire_oldest()

    def poll(self):
        """Retire the rounds that have completed, without waiting."""
        while self._inflight and self._inflight[0][1].query():
            self._retire_oldest()

    def stats(self, since: float | None = None) -> dict:
        reqs = [r for r in self.done if since is None or r.arrival >= since]
        lat = np.array([r.latency for r in reqs]) if reqs else np.zeros(0)
        poses = int(sum(r.n for r in reqs))
        span = (max(r.finished for r in reqs) - min(r.arrival for r in reqs)) if reqs else 0.0
        return {"requests": len(reqs), "poses": poses,
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "poses_per_s": poses / span if span > 0 else None,
                "rounds": self.rounds, "launches": self.launches, "gpu_s": self.gpu_ms / 1e3,
                "pending": len(self.pending), "active": len(self.active)}

    # ------------------------------------------------------------ internals
    def _admit(self, now: float):
        while self.pending:
            req = self.pending[0]
            s = self.pool.alloc(req.n)
            if s < 0:
                break
            self.pending.popleft()
            req.slot0, req.step, req.admitted = s, req.step0, now
            self.pose[s:s + req.n].copy_(torch.from_numpy(np.ascontiguousarray(req.poses, np.float32)),
                                         non_blocking=True)
            if req.adam0 is None:
                self.state[s:s + req.n].zero_()
            else:
                self.state[s:s + req.n].copy_(torch.from_numpy(np.ascontiguousarray(req.adam0, np.float32)))
            self.active.append(req)

    def shape_of(self, n_beads: int) -> tuple[int, int]:
        """(lanes per pose, beads per lane) of a request whose ligand has
        ``n_beads`` beads; the kernel runs ligands beyond 4 beads per lane in
        chunks of 4."""
        return launch_shape(n_beads, int(self.lanes_for(n_beads)))

    def _group(self, shape, reqs):
        """The LigandSet, work counter and stream of one shape group (the
        ligand set rebuilt only when the group's requests changed)."""
        key = tuple(r.rid for r in reqs)
        g = self._groups.get(shape)
        if g is None:
            g = [None, None, torch.zeros(1, dtype=torch.int32, device=self.device),
                 torch.cuda.Stream(self.device) if self.concurrent else None]
            self._groups[shape] = g
        if g[0] != key:
            g[0], g[1] = key, LigandSet([r.ligand for r in reqs], device=self.device)
        return g

    def round(self, now: float | None = None):
        """Retire completed rounds, admit what fits, and enqueue one round that
        advances every active request by round_steps ADAM steps."""
        self.poll()
        now = time.perf_counter() if now is None else now
        torch.cuda.nvtx.range_push("serve.admit")
        self._admit(now)
        torch.cuda.nvtx.range_pop()
        if not self.active:
            if self._inflight:
                self._retire_oldest()
            return
        torch.cuda.nvtx.range_push("serve.round")
        groups = {}
        for r in self.active:
            groups.setdefault(self.shape_of(len(r.ligand[0])), []).append(r)
        main = torch.cuda.current_stream(self.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        # every group's tables first (uploaded on the current stream), then the
        # launches, each group on its own stream, so that the groups overlap;
        # the tables stay referenced until the round is retired
        tables = []
        for shape in sorted(groups, key=lambda sh: (-sh[1], -sh[0])):  # longest tiles first
            reqs = sorted(groups[shape], key=launch_order)
            lig_key, ligs, counter, stream = self._group(shape, reqs)
            segs = [Segment(r.receptor, i, r.n, r.step, r.slot0) for i, r in enumerate(reqs)]
            wl = Workload(self.grids, ligs, segs, shape[0], self.device, n_poses=self.capacity)
            tables.append((shape, wl, ligs, counter, stream))
        for shape, wl, ligs, counter, stream in tables:
            scratch = _GroupScratch(self.scratch, counter)
            launch = LaunchShape(shape[0], self.launch.block_threads, self.launch.blocks, self.launch.test_flags)
            if stream is not None:
                stream.wait_stream(main)
            with torch.cuda.stream(stream if stream is not None else main):
                minimise(wl, self.pose, self.round_steps, self.adam, self.opts, pose_out=self.pose,
                         adam_state=self.state, launch=launch, scratch=scratch)
            self.launches += 1
        for shape, wl, ligs, counter, stream in tables:
            if stream is not None:
                main.wait_stream(stream)
        # requests that finish with this round: results to the pinned mirror,
        # ordered after the round on the current stream; their rows go back to
        # the pool (later writes to them are enqueued after these copies)
        still, finishing = [], []
        for r in self.active:
            r.step += self.round_steps
            (finishing if r.step >= self.steps else still).append(r)
        if finishing:
            rows = [(r.slot0, r.n) for r in finishing]
            # a mirror row that still holds an unretired request's results is
            # retired first (only when a request finishes in its first round)
            while self._inflight and any(_overlap(rows, (q.slot0, q.n)) for q in self._unretired()):
                self._retire_oldest()
            for r in finishing:
                sl = slice(r.slot0, r.slot0 + r.n)
                self.h_pose[sl].copy_(self.pose[sl], non_blocking=True)
                self.h_energy[sl].copy_(self.scratch.energy[sl], non_blocking=True)
                self.h_status[sl].copy_(self.scratch.status[sl], non_blocking=True)
                self.pool.release(r.slot0, r.n)
        e1.record(main)
        self._inflight.append((e0, e1, finishing, tables))
        self.active = still
        self.rounds += 1
        torch.cuda.nvtx.range_pop()
        # with k = max_rounds_in_flight, wait until at most k - 1 rounds are
        # outstanding: k = 2 keeps this round queued while the host prepares
        # the next one; k = 1 is a synchronous loop
        while len(self._inflight) >= self.max_rounds_in_flight:
            self._retire_oldest()

    def _unretired(self):
        for _, _, fin, _ in self._inflight:
            yield from fin

    def _retire_oldest(self):
        """Wait for the oldest enqueued round; retire the requests it finished."""
        torch.cuda.nvtx.range_push("serve.retire")
        e0, e1, finishing, tables = self._inflight.popleft()
        e1.synchronize()
        self.gpu_ms += e0.elapsed_time(e1)
        t = time.perf_counter()
        for r in finishing:
            sl = slice(r.slot0, r.slot0 + r.n)
            r.result_poses = self.h_pose[sl].numpy().copy()
            r.result_energies = self.h_energy[sl].numpy().copy()
            r.result_status = self.h_status[sl].numpy().copy()
            r.finished = t
            self.done.append(r)
            self._log(r)
        del tables
        torch.cuda.nvtx.range_pop()

    def _log(self, r: Request):
        if self.log is None:
            return
        E = r.result_energies
        ok = np.isfinite(E) & (r.result_status == 0)
        rec = {"rid": r.rid, "receptor": r.receptor, "poses": r.n, "beads": int(len(r.ligand[0])),
               "arrival_s": r.arrival - self.t0, "admitted_s": r.admitted - self.t0,
               "finished_s": r.finished - self.t0, "latency_s": r.latency, "queue_s": r.admitted - r.arrival,
               "best_energy": float(E[ok].min()) if ok.any() else None,
               "median_energy": float(np.median(E[ok])) if ok.any() else None,
               "flagged_poses": int((~ok).sum())}
        self.log.write(json.dumps(rec) + "\n")
        self.log.flush()

    # ------------------------------------------------------- checkpointing
    def snapshot(self) -> dict:
        """The unfinished requests, between rounds: per active request its
        current poses, ADAM moments and step; pending requests as submitted.
        Plain NumPy / Python values (``numpy.savez`` / pickle friendly)."""
        self.drain()
        torch.cuda.synchronize(self.device)
        reqs = []
        for r in self.active:
            sl = slice(r.slot0, r.slot0 + r.n)
            reqs.append(dict(receptor=r.receptor, ligand=_lig_copy(r.ligand),
                             poses=self.pose[sl].cpu().numpy(), adam=self.state[sl].cpu().numpy(),
                             step=r.step, rid=r.rid, arrival=r.arrival))
        for r in self.pending:
            reqs.append(dict(receptor=r.receptor, ligand=_lig_copy(r.ligand),
                             poses=np.asarray(r.poses), adam=r.adam0, step=r.step0, rid=r.rid, arrival=r.arrival))
        return {"steps": self.steps, "round_steps": self.round_steps, "requests": reqs}

    @classmethod
    def resume(cls, grids, snap: dict, **kw) -> "DockingServer":
        """A server that continues the requests of ``snap`` (same receptors,
        same step schedule); their results equal an uninterrupted run's."""
        srv = cls(grids, steps=snap["steps"], round_steps=snap["round_steps"], **kw)
        for q in snap["requests"]:
            req = Request(q["receptor"], q["ligand"], q["poses"], adam0=q["adam"], step0=int(q["step"]))
            srv.submit(req, now=q["arrival"])
        return srv


def _overlap(rows, span) -> bool:
    s, n = span
    return any(a < s + n and s < a + m for a, m in rows)


def replay(server: DockingServer, requests, duration: float | None = None, time_scale: float = 1.0,
           pose_source=None):
    """Feed requests (dicts with arrival time ``t``, ``receptor``, ``ligand`` and
    ``poses`` -- or ``n_poses`` drawn from ``pose_source(n)``) to the server in
    wall-clock time (``t * time_scale`` after start) for ``duration`` seconds.
    Returns the server's stats for the requests that arrived in the window and
    finished, plus the number that arrived."""
    t0 = time.perf_counter()
    queue = deque(sorted(requests, key=lambda r: r["t"]))
    arrived = 0
    while True:
        now = time.perf_counter() - t0
        if duration is not None and now > duration:
            break
        while queue and queue[0]["t"] * time_scale <= now:
            q = queue.popleft()
            poses = q["poses"] if "poses" in q else pose_source(q["n_poses"])
            server.submit(Request(q["receptor"], q["ligand"], poses), now=t0 + q["t"] * time_scale)
            arrived += 1
        if server.idle():
            if not queue:
                break
            time.sleep(min(0.001, max(0.0, queue[0]["t"] * time_scale - now)))
            continue
        server.round()
    server.drain()
    st = server.stats(since=t0)
    st["arrived"] = arrived
    st["window_s"] = time.perf_counter() - t0
    st["backlog_requests"] = len(server.pending) + len(server.active)
    st["backlog_poses"] = int(sum(r.n for r in server.pending) + sum(r.n for r in server.active))
    return st
