"""Checkpointed solve (fg_forward_checkpointed + fg_adjoint_reference_checkpointed)
against the full-history solve: the same kernels on recomputed history, so
traces, gradients and norms must agree bit for bit."""
import numpy as np
import pytest
import torch

import helpers

gpu = pytest.mark.gpu

TUNINGS = {
    "default": None,
    "lane_both": dict(lanes=1, cells_per_thread=4, rows_per_tile=4, kernel=1),
    "tiles_both": dict(lanes=1, cells_per_thread=4, rows_per_tile=8, warps_per_block=4, stages=2, kernel=0),
    "lane_fwd_tiles_adj": dict(lanes=1, cells_per_thread=4, rows_per_tile=4, kernel=1, adj_kernel=1,
                               adj_rows_per_tile=4, adj_warps_per_block=2, adj_stages=3),
    "columns": dict(lanes=2),
    "pairs": dict(lanes=3, cells_per_thread=2, rows_per_tile=4, kernel=1),
}


def _solve_both(fg, wl, tuning, interval):
    dev = torch.device("cuda:0")
    setup = helpers.setup_for(wl, dev)
    solve = fg.Solve(dev, setup, tuning=tuning, tv=False)
    p = solve.plan
    er, se, mr = solve.materials(torch.tensor(wl.er), torch.tensor(wl.se), torch.tensor(wl.mr))
    S, nt, nrx = setup.shots, setup.nt, p.nrx
    rng = np.random.default_rng(5)
    resid = torch.tensor(rng.standard_normal((S, nt, nrx)).astype(np.float32) * 1e-3, device=dev)
    out = []
    for mode in ("full", "ckpt"):
        tr = torch.empty((S, nt, nrx), device=dev)
        ge = torch.empty((setup.nx, setup.ny), device=dev)
        gs = torch.empty_like(ge)
        norms = torch.empty(2, dtype=torch.float64, device=dev)
        if mode == "full":
            h = p.new_hist()
            p.forward(er, se, mr, tr, h)
            p.adjoint_reference(er, se, mr, h, resid, ge, gs, norms=norms)
        else:
            ck = p.new_checkpoints(interval)
            seg = p.new_segment(interval)
            seg.fill_(float("nan"))      # nothing may read a segment step before it is recomputed
            p.forward_checkpointed(er, se, mr, tr, ck, interval)
            p.adjoint_reference_checkpointed(er, se, mr, ck, interval, seg, resid, ge, gs, norms=norms)
        torch.cuda.synchronize()
        p.device_check()
        out.append((tr.cpu().numpy(), ge.cpu().numpy(), gs.cpu().numpy(), norms.cpu().numpy()))
    return out


@gpu
@pytest.mark.parametrize("name", list(TUNINGS))
@pytest.mark.parametrize("interval", [1, 7, 40, 1000])
def test_checkpointed_equals_full_history(fg, name, interval):
    wl = fg.workloads.small(shots=9 if name != "columns" else 3, nt=120, nx=64, ny=56, fixed=True)
    wl.source_step = [0.05, 0.02, 0.0]
    full, ck = _solve_both(fg, wl, TUNINGS[name], interval)
    for a, b, what in zip(full, ck, ("traces", "grad_eps", "grad_sig", "norms")):
        assert np.array_equal(a, b), what


@gpu
def test_checkpoint_keyword_through_compute(fg):
    dev = torch.device("cuda:0")
    wl = fg.workloads.small(shots=3, nt=100)
    res = []
    for ckp in (None, 9, True, "auto"):
        er = torch.tensor(wl.er[:, :, None], device=dev, requires_grad=True)
        se = torch.tensor(wl.se[:, :, None], device=dev, requires_grad=True)
        traces, _ = fg.compute(**wl.kwargs(dev, er=er, se=se, tv=False, checkpoint=ckp))
        (traces ** 2).sum().backward()
        torch.cuda.synchronize()
        res.append((traces.detach().cpu().numpy(), er.grad.cpu().numpy(), se.grad.cpu().numpy()))
    for other in res[1:]:
        for a, b in zip(res[0], other):
            assert np.array_equal(a, b)


@gpu
def test_autotuned_interval_fits_the_budget(fg):
    """autotune_checkpoint: a candidate interval whose checkpoints plus one
    history segment fit the budget; the smallest-footprint interval when
    none does."""
    from importlib import import_module
    at = import_module(helpers.PKG + ".autotune")
    dev = torch.device("cuda:0")
    wl = fg.workloads.small(shots=9, nt=300, nx=64, ny=56, fixed=True)
    wl.source_step = [0.05, 0.02, 0.0]
    setup = helpers.setup_for(wl, dev)
    plan = fg.Solve(dev, setup, tv=False, bind=False).plan
    k = at.autotune_checkpoint(dev, setup, probe_steps=64)
    assert k in at.CKPT_CANDIDATES
    budget = plan.workspace_bytes + at.checkpoint_memory(plan, 32)
    k2 = at.autotune_checkpoint(dev, setup, budget=budget, probe_steps=64)
    assert plan.workspace_bytes + at.checkpoint_memory(plan, k2) <= budget
    k3 = at.autotune_checkpoint(dev, setup, budget=1)
    assert k3 == import_module(helpers.PKG + ".compute").checkpoint_interval(plan, True)
