"""Drop-in ``compute()`` for the reference's src/compute.py.

Same signature and return convention as the reference entry point
(src/compute.py:33-50): ``compute(device, dx, ny, nx, nz, source,
source_apmlitudes, step, er, se, mr, nsrc, nrx, ...)`` returns
``(traces, dt)`` with ``traces`` the Ez receiver traces of shape
(step, iterations, nrx), float32 on the device, differentiable with respect
to ``er`` and ``se`` through a ``torch.autograd.Function`` whose backward is
the reference's gradient convention (src/compute.py:893-942): the reversed
forward operator, the imaging sums normalised to unit L2 norm, plus
``tv_weight * 2 * (m - TV(m))`` when ``tv`` is set.

The time stepping, CPML, sources, receivers, history and imaging all run in
libfastgpr (CUDA, sm_100a) through the C ABI; this module only prepares the
geometry (grid.py) and owns the tensors.  There is no CPU path.

New keywords (after the reference's own, all defaulting to the reference's
behaviour): ``adjoint`` ('reference'), ``tv_weight`` (0.01, the constant of
src/compute.py:920,928) and ``tuning`` (launch shape, see autotune).

``adjoint='exact'`` swaps the reference's gradient for the exact discrete
adjoint of the forward loop (fg_adjoint_exact): the true derivative of the
loss with respect to ``er`` and ``se`` (CPML profile held fixed), not
normalised; the TV term is still added when ``tv`` is set.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import _native
from .grid import SolveSetup, build_setup
from .multiscale import apply_filter
from .tv import total_variation


def _model2d(t: torch.Tensor, nx: int, ny: int) -> torch.Tensor:
    """(nx, ny) float32 contiguous view of a (nx, ny[, 1]) model tensor."""
    t = t.detach()
    if t.dim() == 3:
        if t.shape[2] < 1:
            raise ValueError("model has an empty z axis")
        t = t[:, :, 0]
    if tuple(t.shape[:2]) != (nx, ny):
        raise ValueError("model shape %s does not match the grid (%d, %d)" % (tuple(t.shape), nx, ny))
    return t.to(torch.float32).contiguous()


class Checkpoints:
    """What a checkpointed forward solve keeps for its gradient: the state at
    the start of every `interval`-th step (fg_forward_checkpointed)."""

    def __init__(self, buf: torch.Tensor, interval: int):
        self.buf = buf
        self.interval = interval


def checkpoint_interval(plan, checkpoint) -> Optional[int]:
    """None (keep the whole Ez history) or the checkpoint interval in steps.
    checkpoint=True picks the interval that minimises checkpoints + one
    segment of history; an int is taken as the interval."""
    if checkpoint is None or checkpoint is False:
        return None
    nt = plan.nt
    if checkpoint is True:
        step = plan.hist_floats // nt * 4
        best = None
        for k in range(1, nt + 1):
            mem = plan.checkpoint_bytes(k) + k * step
            if best is None or mem < best[0]:
                best = (mem, k)
            if k * step > best[0]:
                break
        return best[1]
    k = int(checkpoint)
    if k < 1:
        raise ValueError("checkpoint interval must be >= 1")
    return min(k, nt)


class Solve:
    """One planned forward/adjoint solve: geometry, plan and workspace."""

    def __init__(self, device, setup: SolveSetup, tuning: Optional[dict] = None, tv: bool = True,
                 tv_weight: float = 0.01, adjoint: str = "reference", checkpoint=None, bind: bool = True):
        if adjoint not in ("reference", "exact"):
            raise ValueError("adjoint must be 'reference' or 'exact'")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("the FDTD solver runs on CUDA devices only (got %s)" % self.device)
        self.setup = setup
        self.tv = tv
        self.tv_weight = tv_weight
        self.adjoint = adjoint
        s = setup
        if isinstance(tuning, str):
            if tuning != "auto":
                raise ValueError("tuning must be a dict, None or 'auto'")
            from .autotune import autotune
            ones = torch.ones((s.nx, s.ny), dtype=torch.float32, device=self.device)
            tuning = autotune(self.device, s, 4 * ones, 1e-3 * ones, ones)
        self.tuning = tuning
        pml = s.profile.packed() if s.profile is not None else None
        self.plan = _native.Plan(s.nx, s.ny, s.shots, s.nt, s.th, s.dx, s.dt32,
                                 s.src.cpu().numpy(), s.rx.cpu().numpy(), s.srcw, pml, self.device, tuning,
                                 bind=bind)
        if isinstance(checkpoint, str):
            if checkpoint != "auto":
                raise ValueError("checkpoint must be None, True, an interval or 'auto'")
            from .autotune import autotune_checkpoint
            checkpoint = autotune_checkpoint(self.device, s, tuning=tuning)
        self.interval = checkpoint_interval(self.plan, checkpoint)
        if adjoint == "exact" and self.interval is not None:
            raise ValueError("adjoint='exact' keeps the whole Ez history (checkpoint=None)")

    def materials(self, er, se, mr):
        s = self.setup
        return (_model2d(er, s.nx, s.ny).to(self.device), _model2d(se, s.nx, s.ny).to(self.device),
                _model2d(mr, s.nx, s.ny).to(self.device))

    def forward(self, er, se, mr, keep_history: bool = True):
        s = self.setup
        er32, se32, mr32 = self.materials(er, se, mr)
        traces = torch.empty((s.shots, s.nt, self.plan.nrx), dtype=torch.float32, device=self.device)
        if keep_history and self.interval is not None:
            ck = self.plan.new_checkpoints(self.interval)
            self.plan.forward_checkpointed(er32, se32, mr32, traces, ck, self.interval)
            return traces, Checkpoints(ck, self.interval)
        hist = self.plan.new_hist() if keep_history else None
        self.plan.forward(er32, se32, mr32, traces, hist)
        return traces, hist

    def gradient(self, er, se, mr, hist, resid, need_eps=True, need_sig=True, normalize=True):
        s = self.setup
        er32, se32, mr32 = self.materials(er, se, mr)
        resid = resid.detach().to(device=self.device, dtype=torch.float32).contiguous()
        if tuple(resid.shape) != (s.shots, s.nt, self.plan.nrx):
            raise ValueError("residual shape %s != (%d, %d, %d)" % (tuple(resid.shape), s.shots, s.nt, self.plan.nrx))
        ge = torch.empty((s.nx, s.ny), dtype=torch.float32, device=self.device) if need_eps else None
        gs = torch.empty((s.nx, s.ny), dtype=torch.float32, device=self.device) if need_sig else None
        if self.adjoint == "exact":
            self.plan.adjoint_exact(er32, se32, mr32, hist, resid, ge, gs)
        elif isinstance(hist, Checkpoints):
            seg = self.plan.new_segment(hist.interval)
            self.plan.adjoint_reference_checkpointed(er32, se32, mr32, hist.buf, hist.interval, seg, resid, ge, gs,
                                                     normalize=normalize)
        else:
            self.plan.adjoint_reference(er32, se32, mr32, hist, resid, ge, gs, normalize=normalize)
        return ge, gs


class GPRFWI(torch.autograd.Function):
    """Autograd node of one solve (the reference's GPRFWI, compute.py:877-942)."""

    @staticmethod
    def forward(ctx, solve: Solve, er, se, mr):
        ctx.save_for_backward(er, se, mr)
        ctx.solve = solve
        traces, hist = solve.forward(er, se, mr, keep_history=True)
        ctx.hist = hist
        if torch.isnan(traces).any():
            print("⚠️ rxs_gpu contains NaN!")
        return traces

    @staticmethod
    def backward(ctx, grad_output):
        if torch.isnan(grad_output).any():
            print("⚠️ grad_output contains NaN!")
        er, se, mr = ctx.saved_tensors
        solve: Solve = ctx.solve
        need_e, need_s = ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        ge, gs = solve.gradient(er, se, mr, ctx.hist, grad_output, need_e, need_s)
        ctx.hist = None
        if ge is not None:
            ge = ge.view(er.shape)
        if gs is not None:
            gs = gs.view(se.shape)
        if solve.tv:
            lam = solve.tv_weight
            if need_e:
                uer = total_variation(er.detach().clone())
                ge += lam * (2 * (er.detach() - uer))
                if torch.isnan(ge).any():
                    print("⚠️ epsilon.grad contains NaN!")
            if need_s:
                use = total_variation(se.detach().clone())
                gs += lam * (2 * (se.detach() - use))
                if torch.isnan(gs).any():
                    print("⚠️ sigma.grad contains NaN!")
        return None, ge, gs, None


def compute(device, dx, ny, nx, nz, source, source_apmlitudes, step, er, se, mr, nsrc, nrx,
            time_windows=None, source_location=None, source_step=None,
            receiver_location=None, receiver_step=None, pmlthick=0, freq=None,
            dt=None, pml_formulation='HORIPML', total_step=None, tv=True,
            Fixedreceiver=False, nseg=None, customsource=None, customreceiver=None,
            adjoint='reference', tv_weight=0.01, tuning=None, checkpoint=None):
    """Forward-model GPR traces; differentiable w.r.t. ``er`` and ``se``.

    Arguments and return value as the reference's compute() (src/compute.py:33-50).
    ``nseg`` (the reference's history-segmenting switch) does not change the
    result and is accepted for compatibility.  ``checkpoint`` (not in the
    reference): None keeps the whole Ez history for the gradient, as the
    reference does; an int K keeps the solver state every K steps instead and
    recomputes the history segment by segment during the backward pass (one
    extra forward solve, same results bit for bit); True picks the K of the
    smallest footprint; 'auto' the K of the fastest checkpointed gradient
    that fits in 80% of the free device memory, measured on a truncated run
    (autotune.autotune_checkpoint, cached per geometry).
    ``tuning`` (not in the reference): None = default launch shapes, a dict of
    fg_tuning fields, or 'auto' = the fastest shapes for this geometry
    measured on a truncated run (autotune.py, cached per geometry).
    """
    if pml_formulation != 'HORIPML':
        raise ValueError("only the HORIPML formulation is implemented (as in the reference)")
    se = torch.clamp(se, min=0)
    er = torch.clamp(er, min=1)
    setup = build_setup(device, dx, ny, nx, nz, time_windows, source, source_location, source_step,
                        receiver_location, receiver_step, pmlthick, source_apmlitudes, step, er, mr,
                        nsrc, nrx, dt, freq, total_step, Fixedreceiver, customsource, customreceiver)
    # The reference filters the source wavelet here and discards the result
    # (compute.py:825-826); the call is kept for its argument checking.
    if freq is not None and freq != source_apmlitudes[2]:
        apply_filter(torch.from_numpy(setup.srcw[0].copy()), 1 / dt, freq)
    solve = Solve(device, setup, tuning=tuning, tv=tv, tv_weight=tv_weight, adjoint=adjoint, checkpoint=checkpoint)
    traces = GPRFWI.apply(solve, er, se, mr)
    return traces, setup.dt
