"""The inversion loop of the reference's example (example.ipynb, the training
cell): Adam on eps_r (and, after a first phase, sigma), an L1 misfit times a
weight, gradients zeroed on the CPML columns, the TV term of the default
gradient.  Each epoch is one forward solve and one adjoint solve; the plan is
built once, and when the model's first row changes (the HORIPML profile
averages it, grid.slab_average) only its CPML profile is replaced -- the
reference rebuilds its grid, PML profile and coefficient arrays in every
compute() call -- and the L1
misfit's derivative is formed
inside the adjoint's injection (fg_adjoint_reference_l1), so the residual
tensor torch's L1Loss backward would build is never materialised.

With the same inputs an epoch produces the gradients the notebook's
compute() + L1Loss + backward() produce (tests/test_gpu_fwi.py).

checkpoint (an interval, True or 'auto', as compute()'s) keeps the solver
state every K steps instead of the whole Ez history and recomputes the
history segment by segment in the adjoint; the L1 derivative is then formed
by three tensor operations (the same float32 values) and injected as a
residual.  Results equal the full-history epoch's bit for bit.

graph='epoch' captures the whole epoch -- clamps, coefficient kernels,
solve, loss, the TV kernel, the clamps' backward, border zeroing and the
Adam step (capturable Adam) -- and replays it; only the loss and row 0 of
eps_r (to see whether the CPML profile changed; when it did, the new profile
is uploaded before the replay) come back to the host.  It
computes the bits of the eager epoch with adam_capturable=True.  Capturable
Adam keeps its step count on the device and arranges the bias corrections
and eps differently from the default Adam, so cells whose gradient is near
eps move differently from the notebook's loop.

graph=True captures an epoch's solve -- the coefficient kernels, state
resets, 2 nt - 1 step launches and the gradient reductions -- in a CUDA graph
with static model, trace and gradient buffers, and replays it every epoch
after copying the current models in (a new CPML profile is written into
the plan's workspace before the replay, so the capture stays valid).
Replays compute the eager solve's bits.
"""
from __future__ import annotations

from typing import Optional, Sequence

import torch

from .compute import Solve
from .grid import build_setup
from .tv import total_variation


class Inversion:
    """Full-waveform inversion of (eps_r, sigma) from observed traces.

    ``kwargs`` are compute()'s keyword arguments for the survey geometry
    (dx, ny, nx, nz, source, source_apmlitudes, step, nsrc, nrx,
    time_windows, source/receiver locations and steps, pmlthick, dt,
    Fixedreceiver); er0/se0/mr are (nx, ny, 1) starting models.  The
    notebook's settings are the defaults: phase 1 (eps_r alone, lr 0.2) for
    50 epochs, then eps_r at lr 0.1 and sigma at lr 1e-4, loss weight 100.
    """

    def __init__(self, device, kwargs: dict, observed: torch.Tensor, er0: torch.Tensor, se0: torch.Tensor,
                 mr: torch.Tensor, phase1_epochs: int = 50, lr: Sequence[float] = (0.2, 0.1, 1e-4),
                 loss_weight: float = 100.0, tv: bool = True, tv_weight: float = 0.01,
                 tuning: Optional[dict] = None, graph=False, checkpoint=None, adam_capturable: bool = False):
        self.device = torch.device(device)
        kw = dict(kwargs)
        self.pml = int(kw.get("pmlthick", 0))
        self.er = er0.detach().clone().to(self.device).requires_grad_(True)
        self.se = se0.detach().clone().to(self.device).requires_grad_(True)
        self.mr = mr.detach().to(self.device)
        self.observed = observed.detach().to(self.device, torch.float32).contiguous()
        self.loss_weight = float(loss_weight)
        self.phase1_epochs = int(phase1_epochs)
        if graph not in (False, True, "epoch"):
            raise ValueError("graph must be False, True or 'epoch'")
        self.graph_epoch = graph == "epoch"
        cap = bool(adam_capturable) or self.graph_epoch
        self.opt1 = torch.optim.Adam([{"params": self.er, "lr": lr[0]}], capturable=cap)
        self.opt2 = torch.optim.Adam([{"params": self.er, "lr": lr[1]}, {"params": self.se, "lr": lr[2]}],
                                     capturable=cap)
        self.kw = kw
        self.solve_args = dict(tuning=tuning, tv=tv, tv_weight=tv_weight, checkpoint=checkpoint)
        self.use_graph = graph is True
        self._graph = None
        self._plan_gen = 0         # plans built so far
        self._egraph = {}          # phase (False/True) -> the whole epoch captured (graph='epoch')
        self._loss = torch.zeros((), dtype=torch.float32, device=self.device)
        self._row0 = None
        self._plan_for(torch.clamp(self.er.detach(), min=1))
        setup = self.setup
        if tuple(self.observed.shape) != (setup.shots, setup.nt, self.solve.plan.nrx):
            raise ValueError("observed traces %s != (%d, %d, %d)" % (tuple(self.observed.shape), setup.shots,
                                                                      setup.nt, self.solve.plan.nrx))
        # torch's L1Loss(mean) * w backward: w / numel in float32, times sign(syn - obs)
        n = torch.tensor(float(self.observed.numel()), dtype=torch.float32)
        self.scale = float(torch.tensor(self.loss_weight, dtype=torch.float32) / n)
        self.epochs = 0

    def _plan_for(self, er_c: torch.Tensor) -> None:
        """Keep the set-up and plan in step with the model: the CPML profile
        is the one part that depends on it (HORIPML averages row 0 of the
        clamped eps_r).  When row 0 changes, the new set-up's profile is
        written into the existing plan (fg_plan_set_profile): its tables,
        buffers and captured graphs stay valid.  The first call builds it."""
        row0 = er_c[0].detach()
        if self._row0 is not None and torch.equal(row0, self._row0):
            return
        kw = self.kw
        setup = build_setup(self.device, kw["dx"], kw["ny"], kw["nx"], kw.get("nz", 1), kw.get("time_windows"),
                            kw["source"], kw.get("source_location"), kw.get("source_step"),
                            kw.get("receiver_location"), kw.get("receiver_step"), kw.get("pmlthick", 0),
                            kw["source_apmlitudes"], kw["step"], er_c.detach(), self.mr, kw["nsrc"], kw["nrx"],
                            kw.get("dt"), kw.get("freq"), kw.get("total_step"), kw.get("Fixedreceiver", False),
                            kw.get("customsource"), kw.get("customreceiver"))
        self._row0 = row0.clone()
        if self._plan_gen > 0:
            if setup.profile is not None:
                self.solve.plan.set_profile(setup.profile.packed())
            self.setup = self.solve.setup = setup
            return
        self.setup = setup
        self.solve = Solve(self.device, self.setup, **self.solve_args)
        self._plan_gen += 1
        self._graph = None
        s, p = self.setup, self.solve.plan
        # static buffers of the solve (the graph's inputs and outputs)
        self._e32 = torch.empty((s.nx, s.ny), dtype=torch.float32, device=self.device)
        self._s32 = torch.empty_like(self._e32)
        self._m32 = self.solve.materials(self.mr, self.mr, self.mr)[2]
        self._traces = torch.empty((s.shots, s.nt, p.nrx), dtype=torch.float32, device=self.device)
        k = self.solve.interval
        if k is None:
            self._hist = p.new_hist()
        else:
            # checkpoints every k steps, one history segment, the L1 derivative
            self._hist = None
            self._ck = p.new_checkpoints(k)
            self._seg = p.new_segment(k)
            self._resid = torch.empty_like(self._traces)
        self._ge = torch.empty((s.nx, s.ny), dtype=torch.float32, device=self.device)
        self._gs = torch.empty_like(self._ge)

    def _solve_into_static(self) -> None:
        """Forward + fused L1 adjoint on the static buffers (eagerly or as a graph replay)."""
        p = self.solve.plan

        k = self.solve.interval

        def run():
            if k is None:
                p.forward(self._e32, self._s32, self._m32, self._traces, self._hist)
                p.adjoint_reference_l1(self._e32, self._s32, self._m32, self._hist, self._traces, self.observed,
                                       self.scale, self._ge, self._gs)
                return
            p.forward_checkpointed(self._e32, self._s32, self._m32, self._traces, self._ck, k)
            # scale * sign(syn - obs) in float32, the value the fused injection forms
            torch.sub(self._traces, self.observed, out=self._resid)
            torch.sign(self._resid, out=self._resid)
            self._resid.mul_(self.scale)
            p.adjoint_reference_checkpointed(self._e32, self._s32, self._m32, self._ck, k, self._seg, self._resid,
                                             self._ge, self._gs)

        if not self.use_graph:
            run()
            return
        if self._graph is None:
            side = torch.cuda.Stream(self.device)
            side.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(side):
                run()                                  # warm-up: launch shapes and occupancy are cached here
            torch.cuda.current_stream(self.device).wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                run()
            self._graph = g
        self._graph.replay()

    def _epoch_body(self, phase2: bool) -> None:
        """The epoch of graph='epoch', without autograd: the clamps' backward
        is where(m >= bound, g, 0), as torch's clamp backward forms it, and
        the gradients are written into the parameters' .grad tensors."""
        opt = self.opt2 if phase2 else self.opt1
        er_c = torch.clamp(self.er.detach(), min=1)
        se_c = torch.clamp(self.se.detach(), min=0)
        e32, s32, _ = self.solve.materials(er_c, se_c, self.mr)
        self._e32.copy_(e32)
        self._s32.copy_(s32)
        self._solve_into_static()
        self._loss.copy_((self._traces - self.observed).abs().mean() * self.loss_weight)
        zero = torch.zeros((), dtype=torch.float32, device=self.device)
        p = self.pml
        pairs = [(self.er, er_c, self._ge, 1)] + ([(self.se, se_c, self._gs, 0)] if phase2 else [])
        for param, m_c, g_static, bound in pairs:
            g = g_static.view(m_c.shape)
            if self.solve.tv:
                tv = total_variation(m_c.clone(), capturable=True)
                g = g + self.solve.tv_weight * (2 * (m_c - tv))
            g = torch.where(param.detach() >= bound, g, zero)
            if p > 0:
                g[:, :p, :] = 0
                g[:, -p:, :] = 0
            param.grad.copy_(g)
        opt.step()

    def _epoch_graphed(self) -> float:
        """graph='epoch': the first epoch of each phase (and the first after a
        plan rebuild) runs eagerly and is then captured; later epochs replay
        the capture.  Only the loss and row 0 of eps_r come back to the host."""
        phase2 = self.epochs >= self.phase1_epochs
        gen = self._plan_gen
        self._plan_for(torch.clamp(self.er.detach(), min=1))
        if self._plan_gen != gen:
            self._egraph = {}                      # new static buffers: capture again
        for param in (self.er, self.se):
            if param.grad is None:
                param.grad = torch.zeros_like(param)
        g = self._egraph.get(phase2)
        if g is None:
            cur = torch.cuda.current_stream(self.device)
            side = torch.cuda.Stream(self.device)
            side.wait_stream(cur)
            with torch.cuda.stream(side):
                self._epoch_body(phase2)           # this epoch, eagerly (creates the optimiser state)
            cur.wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._epoch_body(phase2)           # recorded, not run
            self._egraph[phase2] = g
        else:
            g.replay()
        self.epochs += 1
        return float(self._loss)

    def epoch(self) -> float:
        """One epoch: forward, loss, fused adjoint, border zeroing, Adam step.
        Returns the loss (L1 mean times the weight)."""
        if self.graph_epoch:
            return self._epoch_graphed()
        phase2 = self.epochs >= self.phase1_epochs
        opt = self.opt2 if phase2 else self.opt1
        opt.zero_grad()
        er_c = torch.clamp(self.er, min=1)          # compute() clamps its inputs (autograd keeps the mask)
        se_c = torch.clamp(self.se, min=0)
        self._plan_for(er_c)
        e32, s32, _ = self.solve.materials(er_c.detach(), se_c.detach(), self.mr)
        self._e32.copy_(e32)
        self._s32.copy_(s32)
        self._solve_into_static()
        loss = (self._traces - self.observed).abs().mean() * self.loss_weight
        ge = self._ge.clone().view(er_c.shape)
        gs = self._gs.clone() if phase2 else None
        if self.solve.tv:
            lam = self.solve.tv_weight
            ge = ge + lam * (2 * (er_c.detach() - total_variation(er_c.detach().clone())))
        grads = [ge]
        outs = [er_c]
        if phase2:
            gs = gs.view(se_c.shape)
            if self.solve.tv:
                gs = gs + self.solve.tv_weight * (2 * (se_c.detach() - total_variation(se_c.detach().clone())))
            grads.append(gs)
            outs.append(se_c)
        torch.autograd.backward(outs, grads)
        p = self.pml
        if p > 0:
            self.er.grad[:, :p, :] = 0
            self.er.grad[:, -p:, :] = 0
            if phase2:
                self.se.grad[:, :p, :] = 0
                self.se.grad[:, -p:, :] = 0
        opt.step()
        self.epochs += 1
        return float(loss)
