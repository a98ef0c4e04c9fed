"""Launch-shape autotuner.

The step kernels come in several shapes (lane march or tensor-map tile
pipeline; rows per tile, warps per block, pipeline stages), and which one is
fastest depends on the grid, the shot count and the CPML thickness.  The
autotuner plans the same geometry with a truncated run of `probe_steps`
steps, times the forward step of every forward candidate and the adjoint
step of every adjoint candidate with CUDA events, and returns the fastest
pair as one fg_tuning dict (the adjoint runs on its own plan, so the two are
chosen independently).  Results are cached per (device, grid, shots, CPML
thickness).  Every shape computes the same bits, so tuning changes speed
only.
"""
from __future__ import annotations

import itertools
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from . import _native

_CACHE: Dict[Tuple, dict] = {}

FWD_SHOT = [dict(kernel=1, rows_per_tile=ti) for ti in (2, 4, 6)] + \
           [dict(kernel=0, rows_per_tile=8, warps_per_block=4, stages=s) for s in (2, 3)]
ADJ_SHOT = [dict(adj_kernel=2, adj_rows_per_tile=ti, adj_cells_per_thread=8) for ti in (3, 4, 8)] + \
           [dict(adj_kernel=1, adj_rows_per_tile=8, adj_warps_per_block=4, adj_stages=2, adj_cells_per_thread=4),
            dict(adj_kernel=2, adj_rows_per_tile=4, adj_cells_per_thread=4)]
FWD_COL = [dict(kernel=0, rows_per_tile=ti, warps_per_block=min(ti, 4)) for ti in (4, 8)] + \
          [dict(kernel=1, rows_per_tile=4)]
ADJ_COL = [dict(adj_kernel=1, adj_rows_per_tile=ti, adj_warps_per_block=min(ti, 4)) for ti in (4, 8)] + \
          [dict(adj_kernel=2, adj_rows_per_tile=4)]


def _probe_plan(setup, device, tuning, steps):
    s = setup
    pml = s.profile.packed() if s.profile is not None else None
    return _native.Plan(s.nx, s.ny, s.shots, steps, s.th, s.dx, s.dt32, s.src.cpu().numpy(), s.rx.cpu().numpy(),
                        np.ascontiguousarray(s.srcw[:, :steps]), pml, device, tuning)


def _time_ms(fn, reps):
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    fn()
    best = None
    for _ in range(reps):
        ev[0].record()
        fn()
        ev[1].record()
        torch.cuda.synchronize()
        t = ev[0].elapsed_time(ev[1])
        best = t if best is None else min(best, t)
    return best


def autotune(device, setup, er, se, mr, probe_steps: int = 64, reps: int = 2, lanes: Optional[int] = None) -> dict:
    """The fastest launch shape for this geometry (an fg_tuning dict).
    er/se/mr: (nx, ny) float32 device models (any plausible model will do:
    the kernels' speed does not depend on the values)."""
    device = torch.device(device)
    shot = setup.shots >= 8 if lanes is None else lanes == 1
    key = (torch.cuda.get_device_name(device), setup.nx, setup.ny, setup.shots, setup.th, shot)
    if key in _CACHE:
        return dict(_CACHE[key])
    steps = max(8, min(int(probe_steps), setup.nt))
    base = dict(lanes=1 if shot else 2, cells_per_thread=4 if shot else 2)
    S, nx, ny = setup.shots, setup.nx, setup.ny
    fwd_c, adj_c = (FWD_SHOT, ADJ_SHOT) if shot else (FWD_COL, ADJ_COL)
    best_f = best_a = None
    for f, a in itertools.product(fwd_c, adj_c[:1]):
        tu = dict(base, **f, **a)
        try:
            p = _probe_plan(setup, device, tu, steps)
        except _native.FastGprError:
            continue
        tr = torch.empty((S, steps, p.nrx), device=device)
        h = p.new_hist()
        t = _time_ms(lambda: p.forward(er, se, mr, tr, h), reps)
        if best_f is None or t < best_f[0]:
            best_f = (t, f)
        del p, h
    resid = torch.zeros((S, steps, max(1, int(setup.rx.shape[1]))), device=device)
    for a in adj_c:
        tu = dict(base, **best_f[1], **a)
        try:
            p = _probe_plan(setup, device, tu, steps)
        except _native.FastGprError:
            continue
        tr = torch.empty((S, steps, p.nrx), device=device)
        h = p.new_hist()
        p.forward(er, se, mr, tr, h)
        ge = torch.empty((nx, ny), device=device)
        gs = torch.empty_like(ge)
        t = _time_ms(lambda: p.adjoint_reference(er, se, mr, h, resid[:, :, :p.nrx], ge, gs), reps)
        if best_a is None or t < best_a[0]:
            best_a = (t, a)
        del p, h
    torch.cuda.empty_cache()
    tuning = dict(base, **best_f[1], **best_a[1])
    _CACHE[key] = dict(tuning)
    return tuning


# ---------------------------------------------------------------------------
# Checkpoint interval
# ---------------------------------------------------------------------------
CKPT_CANDIDATES = (4, 8, 16, 32, 64, 128, 256)
_CKPT_CACHE: Dict[Tuple, int] = {}


def checkpoint_memory(plan, interval: int) -> int:
    """Device bytes of a checkpointed gradient at `interval`: the checkpoints
    plus one history segment."""
    return max(0, plan.checkpoint_bytes(interval)) + 4 * interval * (plan.hist_floats // plan.nt)


def autotune_checkpoint(device, setup, tuning=None, budget: Optional[int] = None, probe_steps: int = 512,
                        reps: int = 1) -> int:
    """The checkpoint interval K of the fastest checkpointed gradient
    (fg_forward_checkpointed + fg_adjoint_reference_checkpointed) among the
    candidate intervals whose checkpoints and history segment fit in `budget`
    bytes (default: 80% of the free device memory).

    Each candidate is timed on a truncated run of `probe_steps` steps (at
    least two segments of the largest candidate); its cost per step --
    the checkpoint copies every K steps, the recomputed forward and the
    adjoint, with a segment that stays in L2 or not -- carries over to the
    full run.  Ties within 2% go to the smaller footprint.  Cached per
    (device, grid, shots, nt, CPML, tuning, budget argument)."""
    device = torch.device(device)
    key = (torch.cuda.get_device_name(device), setup.nx, setup.ny, setup.shots, setup.nt, setup.th,
           repr(sorted((tuning or {}).items())), budget)
    if key in _CKPT_CACHE:
        return _CKPT_CACHE[key]
    if budget is None:
        free, _ = torch.cuda.mem_get_info(device)
        budget = int(0.8 * free)
    s = setup
    pml = s.profile.packed() if s.profile is not None else None
    full = _native.Plan(s.nx, s.ny, s.shots, s.nt, s.th, s.dx, s.dt32, s.src.cpu().numpy(), s.rx.cpu().numpy(),
                        s.srcw, pml, device, tuning, bind=False)
    fits = [k for k in CKPT_CANDIDATES if k < s.nt and full.workspace_bytes + checkpoint_memory(full, k) <= budget]
    if not fits:
        # the smallest footprint there is (the interval that minimises it)
        from .compute import checkpoint_interval
        k = checkpoint_interval(full, True)
        _CKPT_CACHE[key] = k
        return k
    steps = min(s.nt, max(int(probe_steps), 2 * max(fits)))
    p = _probe_plan(setup, device, tuning, steps)
    ones = torch.ones((s.nx, s.ny), dtype=torch.float32, device=device)
    er, se, mr = 4 * ones, 1e-3 * ones, ones
    tr = torch.empty((s.shots, steps, p.nrx), device=device)
    resid = torch.zeros_like(tr)
    ge = torch.empty((s.nx, s.ny), device=device)
    gs = torch.empty_like(ge)
    timed = []
    for k in fits:
        ck = p.new_checkpoints(k)
        seg = p.new_segment(k)

        def run():
            p.forward_checkpointed(er, se, mr, tr, ck, k)
            p.adjoint_reference_checkpointed(er, se, mr, ck, k, seg, resid, ge, gs)

        timed.append((_time_ms(run, reps), checkpoint_memory(full, k), k))
        del ck, seg
    del p
    torch.cuda.empty_cache()
    fastest = min(t for t, _, _ in timed)
    k = min((m, k) for t, m, k in timed if t <= 1.02 * fastest)[1]
    _CKPT_CACHE[key] = k
    return k
