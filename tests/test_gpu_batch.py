"""Persistent multi-step solves: the whole time loop of one plan, or of up to
eight plans of different grids, shot counts and step counts, in one
cooperative launch (fg_forward_batch, fg_adjoint_reference_batch and the
persistent single-plan path).  Each model's traces, history and gradients
equal those of the one-launch-per-step path and of the model solved alone,
bit for bit; the persistent forward equals the oracle bit for bit."""
import numpy as np
import pytest
import torch

import helpers

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda:0")


def _models(fg):
    """Uneven models: grid, CPML, shot count and step count all differ."""
    W = fg.workloads
    many = W.small(seed=3, shots=40, nt=200, nx=64, ny=50, pml=5, nrx=6, fixed=True)
    many.source_step = [0.02, 0.01, 0.0]
    return [W.small(), W.config0(), many, W.small(seed=5, shots=1, nt=400, nx=30, ny=70, pml=0, nrx=4)]


def _mats(wl, dev):
    return tuple(torch.tensor(np.ascontiguousarray(a), device=dev) for a in (wl.er, wl.se, wl.mr))


def _weights(solve, seed):
    s = solve.setup
    rng = np.random.default_rng(seed)
    return torch.tensor(rng.standard_normal((s.shots, s.nt, solve.plan.nrx)).astype(np.float32),
                        device=solve.device)


def _alone(solve, mats, w):
    traces, hist = solve.forward(*mats)
    ge, gs = solve.gradient(*mats, hist, w, normalize=False)
    torch.cuda.synchronize()
    return traces, solve.plan.hist_view(hist), ge, gs


def _batch(nat, solves, mats, ws):
    plans = [s.plan for s in solves]
    traces = [torch.full((s.setup.shots, s.setup.nt, s.plan.nrx), float("nan"), device=s.device) for s in solves]
    hists = [s.plan.new_hist() for s in solves]
    nat.forward_batch(plans, [m[0] for m in mats], [m[1] for m in mats], [m[2] for m in mats], traces, hists)
    ge = [torch.full((s.setup.nx, s.setup.ny), float("nan"), device=s.device) for s in solves]
    gs = [torch.full((s.setup.nx, s.setup.ny), float("nan"), device=s.device) for s in solves]
    nat.adjoint_reference_batch(plans, [m[0] for m in mats], [m[1] for m in mats], [m[2] for m in mats], hists,
                                ws, ge, gs, normalize=False)
    torch.cuda.synchronize()
    for p in plans:
        p.device_check()
    return list(zip(traces, [p.hist_view(h) for p, h in zip(plans, hists)], ge, gs))


def _same(a, b, tag):
    names = ("traces", "history", "g_eps", "g_sig")
    for name, x, y in zip(names, a, b):
        assert bool(torch.isfinite(x).all()), "%s not finite: %s" % (name, tag)
        assert torch.equal(x, y), "%s differs: %s" % (name, tag)


@pytest.mark.parametrize("lanes", [1, 2])
def test_persistent_equals_per_step(fg, dev, lanes):
    for k, wl in enumerate(_models(fg)):
        setup = helpers.setup_for(wl, dev)
        mats = _mats(wl, dev)
        one = fg.Solve(dev, setup, tv=False, tuning={"kernel": 1, "lanes": lanes, "persistent": 1})
        per = fg.Solve(dev, setup, tv=False, tuning={"kernel": 1, "lanes": lanes, "persistent": -1})
        w = _weights(one, k)
        _same(_alone(one, mats, w), _alone(per, mats, w), "%s lanes %d" % (wl.name, lanes))


def test_persistent_forward_bit_exact_vs_oracle(fg, orc, dev):
    wl = _models(fg)[3]
    prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
    solve = fg.Solve(dev, setup, tv=False, tuning={"kernel": 1, "lanes": 2, "persistent": 1})
    traces, hist = solve.forward(*_mats(wl, dev))
    o_tr, o_hist = orc.forward(prob, np.float32)
    np.testing.assert_array_equal(traces.cpu().numpy(), o_tr)
    np.testing.assert_array_equal(solve.plan.hist_view(hist).cpu().numpy(), o_hist)


@pytest.mark.parametrize("lanes", [1, 2])
def test_mixed_batch_equals_each_model_alone(fg, dev, lanes):
    nat = helpers.native_mod()
    models = _models(fg)
    solves, mats, ws, alone = [], [], [], []
    for k, wl in enumerate(models):
        s = fg.Solve(dev, helpers.setup_for(wl, dev), tv=False, tuning={"lanes": lanes, "persistent": 1})
        m = _mats(wl, dev)
        w = _weights(s, 10 + k)
        solves.append(s)
        mats.append(m)
        ws.append(w)
        alone.append(_alone(s, m, w))
    # all models in one launch, and a pair in the other order
    for order in (list(range(len(models))), [2, 0]):
        got = _batch(nat, [solves[i] for i in order], [mats[i] for i in order], [ws[i] for i in order])
        for i, r in zip(order, got):
            _same(r, alone[i], "%s in batch %s, lanes %d" % (models[i].name, order, lanes))


def test_batch_rejects_unfit_plans(fg, dev):
    nat = helpers.native_mod()
    models = _models(fg)
    a = fg.Solve(dev, helpers.setup_for(models[0], dev), tv=False, tuning={"lanes": 1, "persistent": 1})
    b = fg.Solve(dev, helpers.setup_for(models[1], dev), tv=False, tuning={"lanes": 2, "persistent": 1})
    c = fg.Solve(dev, helpers.setup_for(models[1], dev), tv=False, tuning={"kernel": 1, "lanes": 1})
    for pair in ((a, b), (a, c)):
        mats = [_mats(models[0], dev), _mats(models[1], dev)]
        traces = [torch.empty((s.setup.shots, s.setup.nt, s.plan.nrx), device=dev) for s in pair]
        with pytest.raises(nat.FastGprError):
            nat.forward_batch([s.plan for s in pair], [m[0] for m in mats], [m[1] for m in mats],
                              [m[2] for m in mats], traces, [None, None])
    with pytest.raises(nat.FastGprError):
        nat.forward_batch([a.plan] * (nat.BATCH_MAX + 1), [None] * 9, [None] * 9, [None] * 9, [None] * 9,
                          [None] * 9)
