"""Serving: continuous batching of forward and gradient solves on one GPU.

Requests (a survey geometry as compute()'s keyword arguments, a model, and
for a gradient the residual at the receivers) arrive at any time.  A request
is admitted as soon as its device footprint fits in what is left of the HBM
budget -- its plans' workspaces, its traces and gradients, and either the
whole Ez history or, when that does not fit, checkpoints plus one history
segment (the checkpointed solve, bit-identical results).  Admitted requests
run side by side, each on a CUDA stream of its own driven by a worker
thread (the library's launches release the GIL), so requests that arrive
while others are on the GPU overlap with them on the device -- except a
request whose steps fill the GPU on their own, which runs alone: a step of
at least EXCLUSIVE_WORK cells x shot groups, or a shot-lane step of at least
SPLIT_WORK, whose step kernels (general, slab and interior beside each other)
are sized for the whole GPU.  Side by side such solves only share the SMs
and the L2, and their early-launched dependent kernels hold SM slots the
other streams could use.  Every result
is computed by the same kernels in the same order as the request alone, so
it is the same alone and in the mix, bit for bit.

Forward requests that share a survey -- the same merge_key, grid, time
axis, source waveform, receiver count and model -- are merged when admitted
into one solve over all their shots (up to MERGE_SHOTS), so a few requests
of a few shots each fill the 32 shot lanes of a warp together instead of
one partly filled solve each; each request gets its own shots' traces, the
bits it gets alone (a shot's result does not depend on the shots beside
it).  Gradient requests are not merged: the imaging sums add the shots of
a shot group together, and a request's gradient must hold its own shots
only.

Small requests in shot lanes (at least 8 shots, a step below SPLIT_WORK)
that queue together -- different grids, models and step counts -- are
batched into one persistent launch per direction (fg_forward_batch and
fg_adjoint_reference_batch, up to 8 requests).  The persistent launch
computes the bits of the launch per step, so each request again gets what
it gets alone.  Larger shot-lane requests are not batched: with the
interior split, one after another they are faster than in one persistent
launch (measured on eight uneven models of 140 x 100 to 296 x 296 cells and
8-32 shots: 20.4 against 15.8 Gcell-steps/s).

Throughput counts a request's nx * ny * shots * nt cell-steps once, forward
or gradient (a forward + adjoint pair counted once, the benchmark's unit).

The reference has no serving path: one compute() call at a time, each
rebuilding its grid.
"""
from __future__ import annotations

import concurrent.futures as cf
import dataclasses
import threading
import time
from dataclasses import dataclass, field
from typing import Hashable, List, Optional

import numpy as np
import torch

from .compute import Solve, checkpoint_interval
from .grid import build_setup


@dataclass
class Request:
    """One solve.  kwargs: compute()'s geometry arguments (no er/se/mr);
    er, se, mr: (nx, ny) or (nx, ny, 1) models; resid: (shots, nt, nrx) for a
    gradient (None: forward only)."""
    kwargs: dict
    er: torch.Tensor
    se: torch.Tensor
    mr: torch.Tensor
    resid: Optional[torch.Tensor] = None
    tuning: Optional[dict] = None
    merge_key: Optional[Hashable] = None   # forward requests of one survey: may share a solve


@dataclass
class Result:
    traces: torch.Tensor
    grad_eps: Optional[torch.Tensor]
    grad_sig: Optional[torch.Tensor]
    cell_steps: int
    bytes_reserved: int
    checkpoint: Optional[int]
    submitted: float = 0.0
    started: float = 0.0
    finished: float = 0.0

    @property
    def latency(self) -> float:
        return self.finished - self.submitted


@dataclass
class _Job:
    req: Request
    fut: cf.Future
    submitted: float
    solve: Optional[Solve] = None
    need: int = 0
    interval: Optional[int] = None
    members: List["_Job"] = field(default_factory=list)   # a merged solve: its requests, in shot order
    slots: int = 0
    work: float = 0.0     # cell-steps the job costs (a gradient 2.5 times its forward)
    batch: bool = False   # members are separate requests solved in one persistent launch


MERGE_SHOTS = 64   # shots of one merged forward solve at most (two groups of 32 shot lanes)

# A solve whose step holds at least this many cells x shot groups keeps the
# whole GPU busy on its own (its persistent launches span every SM), and two
# of them side by side only share the SMs and the L2 (measured: a stream of
# such requests ran at 30 Gcell-steps/s four at a time against 36 one at a
# time).  Such a request runs alone; smaller ones share the GPU.
EXCLUSIVE_WORK = 150_000
# A shot-lane step of at least this many cells x shot groups runs the
# interior split by default (fg_tuning.interior): its general, slab and
# interior kernels are each sized for the whole GPU and launched early
# behind one another, so it too runs alone (measured on a burst of 16 small
# shot-lane gradient and forward requests: 11.6 Gcell-steps/s four at a
# time against 26.6 one at a time).
SPLIT_WORK = 12_000


def _weight(job: "_Job", max_active: int) -> int:
    """Slots a job takes: all of them for a step that fills the GPU, else one."""
    s = job.solve.setup
    shot = s.shots >= 8
    work = s.nx * s.ny * ((s.shots + 31) // 32 if shot else s.shots)
    return max_active if work >= EXCLUSIVE_WORK or (shot and work >= SPLIT_WORK) else 1


def _mergeable(a: "_Job", b: "_Job") -> bool:
    """Two forward requests that may share one solve: same survey key, grid,
    time axis, waveform, receivers and model (checked, not assumed)."""
    ra, rb = a.req, b.req
    if ra.resid is not None or rb.resid is not None or ra.merge_key is None or ra.merge_key != rb.merge_key:
        return False
    if ra.tuning != rb.tuning:
        return False
    sa, sb = a.solve.setup, b.solve.setup
    if (sa.nx, sa.ny, sa.nt, sa.th, sa.dx, sa.dt32) != (sb.nx, sb.ny, sb.nt, sb.th, sb.dx, sb.dt32):
        return False
    if sa.src.shape[1:] != sb.src.shape[1:] or sa.rx.shape[1:] != sb.rx.shape[1:]:
        return False
    if not np.array_equal(sa.srcw, sb.srcw):
        return False
    if (sa.profile is None) != (sb.profile is None) or (
            sa.profile is not None and not np.array_equal(sa.profile.packed(), sb.profile.packed())):
        return False
    return all(torch.equal(torch.as_tensor(x), torch.as_tensor(y)) for x, y in ((ra.er, rb.er), (ra.se, rb.se),
                                                                               (ra.mr, rb.mr)))


BATCH_MAX = 8       # requests of one persistent batch at most (FG_BATCH_MAX)


def _batchable(job: "_Job", max_active: int) -> bool:
    """A request the persistent batch can take: small, shot lanes (the
    default from 8 shots), default launch shape, the whole Ez history on the
    device (no checkpointing)."""
    s = job.solve.setup
    return (not job.members and job.req.tuning is None and s.shots >= 8 and job.interval is None and
            _weight(job, max_active) == 1)


def _setup(device, req: Request):
    kw = req.kwargs
    er = torch.clamp(torch.as_tensor(req.er, device=device, dtype=torch.float32), min=1)
    if er.dim() == 2:
        er = er[:, :, None]
    mr = torch.as_tensor(req.mr, device=device, dtype=torch.float32)
    if mr.dim() == 2:
        mr = mr[:, :, None]
    return build_setup(device, kw["dx"], kw["ny"], kw["nx"], kw.get("nz", 1), kw.get("time_windows"),
                       kw.get("source", ["hertzian", "z"]), kw.get("source_location"), kw.get("source_step"),
                       kw.get("receiver_location"), kw.get("receiver_step"), kw.get("pmlthick", 0),
                       kw["source_apmlitudes"], kw["step"], er, mr, kw["nsrc"], kw["nrx"], kw.get("dt"),
                       kw.get("freq"), kw.get("total_step"), kw.get("Fixedreceiver", False),
                       kw.get("customsource"), kw.get("customreceiver"))


class Server:
    """Admits requests by an HBM budget and runs the admitted ones concurrently.

    hbm_budget: bytes the server may hold on the device (default: 90% of the
    free memory when the server starts); max_active: requests on the GPU at
    once (streams / worker threads); policy: which queued request goes next --
    'sjf' the one with the least work (nx * ny * shots * nt, a gradient
    counted 2.5 times: forward, recomputed or stored history, adjoint),
    unless the oldest has waited max_wait seconds, then the oldest; 'fifo'
    the oldest; merge: merge queued forward requests of one survey; batch:
    solve queued small shot-lane requests together in one persistent launch."""

    def __init__(self, device="cuda:0", hbm_budget: Optional[int] = None, max_active: int = 4,
                 policy: str = "sjf", max_wait: float = 2.0, merge: bool = True, batch: bool = True):
        if policy not in ("sjf", "fifo"):
            raise ValueError("policy must be 'sjf' or 'fifo'")
        self.policy = policy
        self.max_wait = float(max_wait)
        self.merge = bool(merge)
        self.batch = bool(batch)
        self.device = torch.device(device)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(free * 0.9)
        self.budget = int(hbm_budget)
        self.used = 0
        self.max_active = int(max_active)
        self.active = 0
        self.slots = 0      # slots taken by the running jobs (_weight)
        self.peak_active = 0
        self._queue: list = []
        self._lock = threading.Condition()
        self._pool = cf.ThreadPoolExecutor(max_workers=self.max_active)
        self._closed = False
        self.results: list = []
        self.merged = 0     # requests served by a merged forward solve
        self.batched = 0    # requests served by a persistent batch

    # -- admission ----------------------------------------------------------
    def _plan(self, job: _Job) -> None:
        """Host-side plan of a job (no device memory yet) and its footprint."""
        req = job.req
        setup = _setup(self.device, req)
        solve = Solve(self.device, setup, tuning=req.tuning, tv=False, bind=False)
        p = solve.plan
        S, nt, nrx = setup.shots, setup.nt, p.nrx
        fixed = p.workspace_bytes + 4 * S * nt * nrx + (8 * setup.nx * setup.ny if req.resid is not None else 0)
        full = fixed + 4 * p.hist_floats
        job.interval = None
        if req.resid is not None and full > self.budget:
            k = checkpoint_interval(p, True)
            job.interval = k
            full = fixed + max(0, p.checkpoint_bytes(k)) + 4 * k * (p.hist_floats // nt)
        elif req.resid is None:
            full = fixed                            # a forward alone keeps no history
        job.solve = solve
        job.need = full
        job.work = setup.nx * setup.ny * S * nt * (2.5 if req.resid is not None else 1.0)

    def submit(self, req: Request) -> cf.Future:
        """Queue a request; the future resolves to a Result."""
        job = _Job(req, cf.Future(), time.perf_counter())
        self._plan(job)
        if job.need > self.budget:
            job.fut.set_exception(MemoryError("request needs %d bytes, budget %d" % (job.need, self.budget)))
            return job.fut
        with self._lock:
            if self._closed:
                raise RuntimeError("server closed")
            self._queue.append(job)
            self._admit_locked()
        return job.fut

    def _merge_locked(self, job: _Job) -> _Job:
        """A forward job with the queued forward jobs of its survey, as one
        solve over all their shots (the job itself when there is none, or
        when the merged solve would not fit)."""
        if not self.merge or job.req.resid is not None or job.req.merge_key is None:
            return job
        members, shots = [job], job.solve.setup.shots
        for other in list(self._queue):
            if shots + other.solve.setup.shots <= MERGE_SHOTS and _mergeable(job, other):
                members.append(other)
                shots += other.solve.setup.shots
        if len(members) == 1:
            return job
        s0 = job.solve.setup
        setup = dataclasses.replace(s0, shots=shots, src=torch.cat([m.solve.setup.src for m in members]),
                                    rx=torch.cat([m.solve.setup.rx for m in members]))
        solve = Solve(self.device, setup, tuning=job.req.tuning, tv=False, bind=False)
        p = solve.plan
        need = p.workspace_bytes + 4 * shots * setup.nt * p.nrx
        merged = _Job(job.req, cf.Future(), job.submitted, solve, need, None, members)
        if self.used + need > self.budget or self.slots + _weight(merged, self.max_active) > self.max_active:
            return job
        for m in members[1:]:
            self._queue.remove(m)
        return merged

    def _batch_locked(self, job: _Job) -> _Job:
        """A small shot-lane job with the queued ones like it, as one
        persistent batch (the job itself when there is none)."""
        if not self.batch or not _batchable(job, self.max_active):
            return job
        members, need = [job], job.need
        for other in list(self._queue):
            if len(members) == BATCH_MAX:
                break
            if _batchable(other, self.max_active) and self.used + need + other.need <= self.budget:
                members.append(other)
                need += other.need
        if len(members) == 1:
            return job
        for m in members[1:]:
            self._queue.remove(m)
        return _Job(job.req, cf.Future(), job.submitted, None, need, None, members, batch=True)

    def _next_locked(self) -> int:
        """Index of the queued job that goes next (policy)."""
        if self.policy == "fifo" or time.perf_counter() - self._queue[0].submitted > self.max_wait:
            return 0
        return min(range(len(self._queue)), key=lambda i: self._queue[i].work)

    def _admit_locked(self) -> None:
        # the next job (policy) waits until its bytes and its slots fit
        while self._queue:
            i = self._next_locked()
            nxt = self._queue[i]
            if self.slots + _weight(nxt, self.max_active) > self.max_active or self.used + nxt.need > self.budget:
                break
            job = self._batch_locked(self._merge_locked(self._queue.pop(i)))
            job.slots = 1 if job.batch else _weight(job, self.max_active)
            self.slots += job.slots
            self.used += job.need
            self.active += 1
            self.peak_active = max(self.peak_active, self.active)
            self._pool.submit(self._run, job)

    def _release(self, job: _Job) -> None:
        with self._lock:
            self.used -= job.need
            self.slots -= job.slots
            self.active -= 1
            self._admit_locked()
            self._lock.notify_all()

    # -- execution ----------------------------------------------------------
    def _run(self, job: _Job) -> None:
        try:
            started = time.perf_counter()
            stream = torch.cuda.Stream(self.device)
            with torch.cuda.device(self.device), torch.cuda.stream(stream):
                res = self._solve_batch(job) if job.batch else self._solve(job)
                stream.synchronize()
            finished = time.perf_counter()
            job.solve = None
            if job.batch:
                out = []
                for m, r in zip(job.members, res):
                    r.submitted, r.started, r.finished = m.submitted, started, finished
                    out.append((m, r))
            elif job.members:
                # a merged forward: each request takes its own shots' traces
                out, o = [], 0
                for m in job.members:
                    S = m.solve.setup.shots
                    r = dataclasses.replace(res, traces=res.traces[o:o + S].clone(),
                                            cell_steps=res.cell_steps // res.traces.shape[0] * S)
                    o += S
                    r.submitted, r.started, r.finished = m.submitted, started, finished
                    out.append((m, r))
            else:
                res.submitted, res.started, res.finished = job.submitted, started, finished
                out = [(job, res)]
            with self._lock:
                self.results.extend(r for _, r in out)
                if job.batch:
                    self.batched += len(job.members)
                else:
                    self.merged += len(job.members)
            for m, r in out:
                m.fut.set_result(r)
        except Exception as e:   # delivered to the caller(s) through the future(s)
            for m in (job.members or [job]):
                m.fut.set_exception(e)
        finally:
            self._release(job)

    def _solve(self, job: _Job) -> Result:
        req, solve = job.req, job.solve
        p = solve.plan
        p.bind()
        s = solve.setup
        er, se, mr = solve.materials(torch.clamp(torch.as_tensor(req.er, device=self.device), min=1),
                                     torch.clamp(torch.as_tensor(req.se, device=self.device), min=0),
                                     torch.as_tensor(req.mr, device=self.device))
        S, nt, nrx = s.shots, s.nt, p.nrx
        traces = torch.empty((S, nt, nrx), dtype=torch.float32, device=self.device)
        ge = gs = None
        if req.resid is None:
            p.forward(er, se, mr, traces, None)
        else:
            resid = torch.as_tensor(req.resid, device=self.device, dtype=torch.float32).contiguous()
            ge = torch.empty((s.nx, s.ny), dtype=torch.float32, device=self.device)
            gs = torch.empty_like(ge)
            if job.interval is None:
                hist = p.new_hist()
                p.forward(er, se, mr, traces, hist)
                p.adjoint_reference(er, se, mr, hist, resid, ge, gs)
            else:
                ck = p.new_checkpoints(job.interval)
                seg = p.new_segment(job.interval)
                p.forward_checkpointed(er, se, mr, traces, ck, job.interval)
                p.adjoint_reference_checkpointed(er, se, mr, ck, job.interval, seg, resid, ge, gs)
        cells = s.nx * s.ny * S * nt
        return Result(traces, ge, gs, cells, job.need, job.interval)

    def _solve_batch(self, job: _Job) -> list:
        """The batch's requests in one persistent launch per direction, each on
        a persistent plan of its own geometry (fg_forward_batch /
        fg_adjoint_reference_batch)."""
        from . import _native
        dev = self.device
        solves, mats = [], []
        for m in job.members:
            s = Solve(dev, m.solve.setup, tuning={"lanes": 1, "persistent": 1}, tv=False)
            solves.append(s)
            req = m.req
            mats.append(s.materials(torch.clamp(torch.as_tensor(req.er, device=dev), min=1),
                                    torch.clamp(torch.as_tensor(req.se, device=dev), min=0),
                                    torch.as_tensor(req.mr, device=dev)))
        plans = [s.plan for s in solves]
        traces = [torch.empty((s.setup.shots, s.setup.nt, s.plan.nrx), dtype=torch.float32, device=dev)
                  for s in solves]
        grads = [m.req.resid is not None for m in job.members]
        hists = [s.plan.new_hist() if g else None for s, g in zip(solves, grads)]
        col = lambda k: [x[k] for x in mats]
        _native.forward_batch(plans, col(0), col(1), col(2), traces, hists)
        ge = [None] * len(solves)
        gs = [None] * len(solves)
        gi = [k for k, g in enumerate(grads) if g]
        if gi:
            for k in gi:
                s = solves[k].setup
                ge[k] = torch.empty((s.nx, s.ny), dtype=torch.float32, device=dev)
                gs[k] = torch.empty_like(ge[k])
            resid = [torch.as_tensor(job.members[k].req.resid, device=dev, dtype=torch.float32).contiguous()
                     for k in gi]
            _native.adjoint_reference_batch([plans[k] for k in gi], [mats[k][0] for k in gi],
                                            [mats[k][1] for k in gi], [mats[k][2] for k in gi],
                                            [hists[k] for k in gi], resid, [ge[k] for k in gi],
                                            [gs[k] for k in gi])
        out = []
        for k, m in enumerate(job.members):
            s = solves[k].setup
            out.append(Result(traces[k], ge[k], gs[k], s.nx * s.ny * s.shots * s.nt, m.need, None))
        return out

    # -- reporting ----------------------------------------------------------
    def close(self, wait: bool = True) -> None:
        with self._lock:
            self._closed = True
        self._pool.shutdown(wait=wait)

    def stats(self) -> dict:
        """p50 / p99 latency (s) and throughput (Gcell-steps/s) over the results so far."""
        with self._lock:
            res = list(self.results)
        if not res:
            return {}
        lat = np.array([r.latency for r in res])
        span = max(r.finished for r in res) - min(r.submitted for r in res)
        cells = sum(r.cell_steps for r in res)
        return {"requests": len(res), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "throughput_gcs": cells / span / 1e9 if span > 0 else float("nan"),
                "peak_active": self.peak_active, "merged": self.merged, "batched": self.batched}
