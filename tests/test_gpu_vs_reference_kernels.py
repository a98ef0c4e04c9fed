"""The reference's own CUDA kernels (oracle/_ref, driven as its Python driver
drives them) and this library, timed on the same GPU on the same problem:
the 64-shot 440 x 340 benchmark grid with a bounded number of steps.  Both
are timed end to end per fwd + adjoint (reference mode) with inputs resident
on the device, and the throughput of each is printed (pytest -s) in
Gcell-steps/s, the benchmark's metric.  The test asserts that the library
is faster and that the traces agree."""
import time

import numpy as np
import pytest
import torch

import helpers

pytestmark = pytest.mark.gpu

NT = 60


@pytest.fixture(scope="module")
def refdrv():
    from oracle import ref_driver
    if not ref_driver.available():
        pytest.fail("reference kernels not built: run make -C oracle ref")
    return ref_driver


def _time(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return best


def test_library_vs_reference_kernels_same_gpu(fg, refdrv):
    dev = torch.device("cuda:0")
    wl = fg.workloads.config2(shots=64, nt=NT)
    kw = wl.kwargs(dev)
    er = torch.clamp(kw["er"], min=1)
    se = torch.clamp(kw["se"], min=0)
    G = refdrv.setup(dev, kw["dx"], kw["ny"], kw["nx"], 1, kw["time_windows"], kw["source_location"],
                     kw["source_step"], kw["receiver_location"], kw["receiver_step"], kw["pmlthick"],
                     kw["source_apmlitudes"], kw["step"], er, se, kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"],
                     kw["Fixedreceiver"])
    S, nrx = wl.shots, wl.nrx
    rng = np.random.default_rng(4)
    w = torch.tensor(rng.standard_normal((S, NT, nrx)).astype(np.float32) * 1e-3, device=dev)
    ref_out = {}

    def ref_step():
        rxs, hist = refdrv.forward(G)
        ref_out["traces"] = rxs[:, 2].contiguous()
        refdrv.backward(G, er, se, kw["mr"], hist, w)

    setup = helpers.setup_for(wl, dev)
    solve = fg.Solve(dev, setup, tv=False)
    e32, s32, m32 = solve.materials(er, se, kw["mr"])
    plan = solve.plan
    hist = plan.new_hist()
    tr = torch.empty((S, NT, plan.nrx), device=dev)
    ge = torch.empty((wl.nx, wl.ny), device=dev)
    gs = torch.empty_like(ge)

    def our_step():
        plan.forward(e32, s32, m32, tr, hist)
        plan.adjoint_reference(e32, s32, m32, hist, w, ge, gs)

    t_ref = _time(ref_step, reps=2)
    t_our = _time(our_step, reps=3)
    cells = wl.nx * wl.ny * S * NT
    g_ref, g_our = cells / t_ref / 1e9, cells / t_our / 1e9
    print("\nreference kernels: %.3f Gcell-steps/s (%.1f ms per fwd+adj of %d steps); library: %.3f Gcell-steps/s "
          "(%.1f ms); ratio %.1fx" % (g_ref, t_ref * 1e3, NT, g_our, t_our * 1e3, g_our / g_ref))
    assert g_our > g_ref
    a, b = tr.cpu().numpy(), ref_out["traces"].cpu().numpy()
    assert helpers.rel_l2(a, b) < 1e-5
