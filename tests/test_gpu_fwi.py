"""The inversion loop (fg.Inversion: fused L1 adjoint, plan reused while the
CPML profile's input is unchanged) against the reference example's loop
written with the drop-in compute(): L1Loss * 100, backward, border zeroing,
two-phase Adam.  Same losses and models epoch by epoch."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(fg):
    wl = fg.workloads.small(shots=3, nt=100)
    dev = torch.device("cuda:0")
    true_er = torch.tensor(wl.er[:, :, None], device=dev)
    true_se = torch.tensor(wl.se[:, :, None], device=dev)
    er0 = torch.full_like(true_er, float(np.median(wl.er)))
    se0 = torch.full_like(true_se, float(np.median(wl.se)))
    mr = torch.tensor(wl.mr[:, :, None], device=dev)
    with torch.no_grad():
        obs, _ = fg.compute(**wl.kwargs(dev, er=true_er, se=true_se, mr=mr, tv=False))
    return wl, dev, obs.detach(), er0, se0, mr


def _notebook_loop(fg, wl, dev, obs, er0, se0, mr, epochs, phase1):
    er = er0.clone().requires_grad_(True)
    se = se0.clone()
    opt1 = torch.optim.Adam([{"params": er, "lr": 0.2}])
    opt2 = torch.optim.Adam([{"params": er, "lr": 0.1}, {"params": se, "lr": 0.0001}])
    l1 = torch.nn.L1Loss()
    p = wl.pml
    out = []
    for epoch in range(epochs):
        opt = opt1 if epoch < phase1 else opt2
        se.requires_grad = epoch >= phase1
        opt.zero_grad()
        result, _ = fg.compute(**wl.kwargs(dev, er=er, se=se, mr=mr, tv=True))
        loss = l1(result, obs) * 100
        loss.backward()
        er.grad[:, :p, :] = 0
        er.grad[:, -p:, :] = 0
        if se.requires_grad:
            se.grad[:, :p, :] = 0
            se.grad[:, -p:, :] = 0
        opt.step()
        out.append((loss.item(), er.detach().cpu().numpy().copy(), se.detach().cpu().numpy().copy()))
    return out


def test_inversion_matches_notebook_loop(fg):
    wl, dev, obs, er0, se0, mr = _problem(fg)
    epochs, phase1 = 4, 2
    ref = _notebook_loop(fg, wl, dev, obs, er0, se0, mr, epochs, phase1)
    kw = wl.kwargs(dev, tv=True)
    for k in ("er", "se", "mr", "tv", "device"):
        kw.pop(k)
    inv = fg.Inversion(dev, kw, obs, er0, se0, mr, phase1_epochs=phase1)
    for e in range(epochs):
        loss = inv.epoch()
        r_loss, r_er, r_se = ref[e]
        assert abs(loss - r_loss) <= 1e-6 * abs(r_loss), (e, loss, r_loss)
        np.testing.assert_allclose(inv.er.detach().cpu().numpy(), r_er, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(inv.se.detach().cpu().numpy(), r_se, rtol=1e-6, atol=1e-10)


def test_inversion_reduces_misfit(fg):
    wl, dev, obs, er0, se0, mr = _problem(fg)
    kw = wl.kwargs(dev, tv=True)
    for k in ("er", "se", "mr", "tv", "device"):
        kw.pop(k)
    inv = fg.Inversion(dev, kw, obs, er0, se0, mr, phase1_epochs=3)
    losses = [inv.epoch() for _ in range(6)]
    assert losses[-1] < losses[0]


def test_inversion_graph_replay_equals_eager(fg):
    """The epoch's solve captured in a CUDA graph and replayed gives the eager bits."""
    wl, dev, obs, er0, se0, mr = _problem(fg)
    kw = wl.kwargs(dev, tv=True)
    for k in ("er", "se", "mr", "tv", "device"):
        kw.pop(k)
    runs = []
    for graph in (False, True):
        inv = fg.Inversion(dev, kw, obs, er0, se0, mr, phase1_epochs=2, graph=graph)
        losses = [inv.epoch() for _ in range(4)]
        runs.append((losses, inv.er.detach().cpu().numpy(), inv.se.detach().cpu().numpy(), inv._graph is not None))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][2], runs[1][2])
    assert runs[1][3] and not runs[0][3]


def test_inversion_checkpointed_equals_full_history(fg):
    """Checkpointed epochs (state every k steps, L1 derivative as a residual)
    give the full-history epochs' losses and models bit for bit."""
    wl, dev, obs, er0, se0, mr = _problem(fg)
    kw = wl.kwargs(dev, tv=True)
    for k in ("er", "se", "mr", "tv", "device"):
        kw.pop(k)
    runs = []
    for ckp in (None, 7, "auto"):
        inv = fg.Inversion(dev, kw, obs, er0, se0, mr, phase1_epochs=2, checkpoint=ckp)
        losses = [inv.epoch() for _ in range(4)]
        runs.append((losses, inv.er.detach().cpu().numpy(), inv.se.detach().cpu().numpy()))
    for other in runs[1:]:
        assert other[0] == runs[0][0]
        assert np.array_equal(other[1], runs[0][1]) and np.array_equal(other[2], runs[0][2])


def test_inversion_whole_epoch_graph_equals_eager(fg):
    """graph='epoch' (clamps, solve, loss, TV, clamp backward, border zeroing
    and Adam in one CUDA graph, replayed; the CPML profile updated in place as
    row 0 of eps_r changes) gives the eager epochs' bits with the same
    (capturable) Adam.  Capturable Adam divides by its bias corrections in
    another arrangement than the default one, which moves cells whose
    gradient is near Adam's eps, so it is not compared with the notebook's
    default-Adam loop."""
    wl, dev, obs, er0, se0, mr = _problem(fg)
    kw = wl.kwargs(dev, tv=True)
    for k in ("er", "se", "mr", "tv", "device"):
        kw.pop(k)
    runs = []
    for graph in (False, "epoch"):
        inv = fg.Inversion(dev, kw, obs, er0, se0, mr, phase1_epochs=2, graph=graph, adam_capturable=True)
        losses = [inv.epoch() for _ in range(5)]
        runs.append((losses, inv.er.detach().cpu().numpy(), inv.se.detach().cpu().numpy(), len(inv._egraph),
                     inv._plan_gen))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][2], runs[1][2])
    assert runs[1][3] == 2 and runs[1][4] == 1      # one capture per phase, one plan
