"""adjoint='exact' on the GPU (fg_adjoint_exact through the C ABI): the FP32
gradient against the FP64 oracle's exact adjoint, and against centred finite
differences of the FP64 oracle's forward on config 1 (240x160, 13 shots,
nt 3000), with the cosine similarity between the exact and the reference-mode
gradients printed."""
import numpy as np
import pytest
import torch

import helpers

pytestmark = pytest.mark.gpu

TOL = 1e-4   # relative error of the FP32 gradient against FP64 (north_star bound)


@pytest.fixture(scope="module")
def dev():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda:0")


def _exact_gpu(fg, wl, dev, w, tuning=None):
    setup = helpers.setup_for(wl, dev)
    solve = fg.Solve(dev, setup, tv=False, adjoint="exact", tuning=tuning)
    er, se, mr = (torch.tensor(np.ascontiguousarray(a), device=dev) for a in (np.maximum(wl.er, 1),
                                                                              np.maximum(wl.se, 0), wl.mr))
    traces, hist = solve.forward(er, se, mr)
    ge, gs = solve.gradient(er, se, mr, hist, torch.tensor(w, device=dev))
    torch.cuda.synchronize()
    return traces, ge.cpu().numpy().astype(np.float64), gs.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("case,tuning", [
    (0, None), (0, {"lanes": 2}), (1, None), (1, {"lanes": 1}), (2, None), (3, None),
])
def test_exact_vs_fp64_oracle(fg, orc, dev, case, tuning):
    if case == 2:
        # two shot groups on a narrow grid with CPML slabs 8 cells thick
        wl = fg.workloads.small(seed=11, shots=40, nt=90, nx=33, ny=65, pml=8, nrx=5)
        wl.source_step = [0.01, 0.02, 0.0]
        wl.receiver_step = [0.05, 0.0, 0.0]
        wl.fixed_receiver = True
    else:
        wl = [fg.workloads.small(), fg.workloads.small(seed=3, shots=2, nt=150, nx=40, ny=56, pml=5, nrx=6), None,
              fg.workloads.config0()][case]
    rng = np.random.default_rng(31 + case)
    w = rng.standard_normal((wl.shots, wl.nt, wl.nrx)).astype(np.float32)
    _, ge, gs = _exact_gpu(fg, wl, dev, w, tuning)
    prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
    p64 = helpers.fp64_problem(prob, setup, wl)
    _, hist = orc.forward(p64, np.float64)
    s1, s2 = orc.exact_sums(p64, hist, w.astype(np.float64))
    oe, os_ = orc.exact_gradient(s1, s2, np.maximum(wl.er, 1), np.maximum(wl.se, 0), setup.dt32)
    e_ge, e_gs = helpers.rel_l2(ge, oe), helpers.rel_l2(gs, os_)
    print("%s exact adjoint vs FP64 oracle: g_eps %.3g, g_sig %.3g" % (wl.name, e_ge, e_gs))
    assert np.isfinite(ge).all() and np.isfinite(gs).all()
    assert e_ge <= TOL and e_gs <= TOL


def test_exact_vs_centred_fd_config1(fg, orc, dev):
    """Directional derivatives of J = sum w * traces along smooth eps_r and
    sigma perturbations: the GPU's exact gradient against centred FD of the
    FP64 oracle (h = 1e-3 of the parameter's scale), within 1e-4."""
    wl = fg.workloads.config1()
    rng = np.random.default_rng(41)
    w = rng.standard_normal((wl.shots, wl.nt, wl.nrx)).astype(np.float32)
    _, ge, gs = _exact_gpu(fg, wl, dev, w)
    prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
    er = np.maximum(wl.er, 1).astype(np.float64)
    se = np.maximum(wl.se, 0).astype(np.float64)
    w64 = w.astype(np.float64)

    def J(e, s):
        tr, _ = orc.forward(helpers.fp64_problem(prob, setup, wl, e, s), np.float64, keep_history=False)
        return float(np.sum(w64 * tr))

    d = helpers.bump(wl.nx, wl.ny, wl.nx / 2, wl.ny / 2, 12.0)
    for name, de, ds, h in (("eps_r", d, 0 * d, 1e-3 * float(er.mean())),
                            ("sigma", 0 * d, d, 1e-3 * float(se.mean()))):
        fd = (J(er + h * de, se + h * ds) - J(er - h * de, se - h * ds)) / (2 * h)
        ad = float(np.sum(ge * de) + np.sum(gs * ds))
        err = abs(fd - ad) / abs(fd)
        assert np.isfinite(ad)
        print("config1 %s: centred FD %.9g, exact adjoint %.9g, rel err %.3g" % (name, fd, ad, err))
        assert err <= TOL
    # the reference-mode gradient of the same weights, for the cosine similarity of the two modes
    setup_r = helpers.setup_for(wl, dev)
    solve = fg.Solve(dev, setup_r, tv=False)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)
    traces, hist = solve.forward(t(er.astype(np.float32)), t(se.astype(np.float32)), t(wl.mr))
    re_, rs_ = solve.gradient(t(er.astype(np.float32)), t(se.astype(np.float32)), t(wl.mr), hist, t(w))
    cos = lambda a, b: float(np.sum(a * b) / (np.linalg.norm(a) * np.linalg.norm(b)))
    print("config1 cosine(reference mode, exact): g_eps %.4f, g_sig %.4f"
          % (cos(re_.cpu().numpy().astype(np.float64), ge), cos(rs_.cpu().numpy().astype(np.float64), gs)))


def test_compute_exact_autograd(fg, dev):
    """compute(..., adjoint='exact') backward == Solve.gradient of the same weights."""
    wl = fg.workloads.small(shots=4, nt=100)
    rng = np.random.default_rng(7)
    w = rng.standard_normal((wl.shots, wl.nt, wl.nrx)).astype(np.float32)
    er = torch.tensor(np.maximum(wl.er, 1)[:, :, None], device=dev, requires_grad=True)
    se = torch.tensor(np.maximum(wl.se, 0)[:, :, None], device=dev, requires_grad=True)
    traces, _ = fg.compute(**wl.kwargs(dev, er=er, se=se, tv=False, adjoint="exact"))
    (traces * torch.tensor(w, device=dev)).sum().backward()
    _, ge, gs = _exact_gpu(fg, wl, dev, w)
    assert np.array_equal(er.grad[:, :, 0].cpu().numpy().astype(np.float64), ge)
    assert np.array_equal(se.grad[:, :, 0].cpu().numpy().astype(np.float64), gs)
