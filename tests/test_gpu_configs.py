"""Parity on the benchmark configurations and on edge shapes.

  - config 1 (240x160, 13 shots, nt 3000): traces and both reference-mode
    gradients against the reference's own CUDA kernels (oracle/ref_driver.py),
    and against the FP64 oracle over its first 1000 steps;
  - a config-2 sample (440x340, all 64 shots, 1000 steps -- long enough for
    the forward and adjoint fields to meet between the source and receiver
    boreholes, so the gradient is not zero): traces and
    gradients against the reference's kernels, for the default launch shape
    and the band pipeline;
  - every grid nx, ny in {17, 33, 65} with CPML 0, 1 and 8 cells, through the
    bounds-checked build (tests/checked_edge_shapes.py, its own process);
  - the fused L1 adjoint (fg_adjoint_reference_l1) against the oracle's
    reference adjoint fed with scale * sign(traces - observed).
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import helpers

pytestmark = pytest.mark.gpu

TOL_REF = 1e-5
TOL_FP64 = 1e-4
HERE = os.path.dirname(os.path.abspath(__file__))
BAND = {"lanes": 1, "kernel": 2, "cells_per_thread": 4, "warps_per_block": 4, "rows_per_tile": 8, "stages": 4,
        "adj_kernel": 3, "adj_cells_per_thread": 4, "adj_rows_per_tile": 8, "adj_stages": 4}


@pytest.fixture(scope="module")
def dev():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda:0")


@pytest.fixture(scope="module")
def refdrv():
    from oracle import ref_driver
    if not ref_driver.available():
        pytest.fail("reference kernels not built: run make -C oracle ref")
    return ref_driver


def _vs_reference(fg, refdrv, wl, dev, tuning=None, seed=17):
    rng = np.random.default_rng(seed)
    w = torch.tensor(rng.standard_normal((wl.shots, wl.nt, wl.nrx)).astype(np.float32), device=dev)
    tr, ge, gs = helpers.run_package(fg, wl, dev, w, tuning=tuning)
    _, rtr, rge, rgs = helpers.run_reference(refdrv, wl, dev, w)
    errs = [helpers.rel_l2(a.cpu().numpy(), b.cpu().numpy()) for a, b in ((tr, rtr), (ge, rge), (gs, rgs))]
    print("%s (%s) vs reference kernels: traces %.3g, g_eps %.3g, g_sig %.3g" % (wl.name, tuning, *errs))
    assert all(np.isfinite(e) for e in errs) and ge.abs().max() > 0 and gs.abs().max() > 0
    return errs


def test_config1_vs_reference_kernels(fg, dev, refdrv):
    errs = _vs_reference(fg, refdrv, fg.workloads.config1(), dev)
    assert max(errs) <= TOL_REF


def test_config1_vs_fp64_oracle(fg, orc, dev):
    wl = fg.workloads.config1()
    wl.nt = 1000
    rng = np.random.default_rng(23)
    w = rng.standard_normal((wl.shots, wl.nt, wl.nrx)).astype(np.float32)
    tr, ge, gs = helpers.run_package(fg, wl, dev, torch.tensor(w, device=dev))
    prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
    p64 = helpers.fp64_problem(prob, setup, wl)
    o_tr, o_hist = orc.forward(p64, np.float64)
    oe, os_ = orc.adjoint_reference(p64, o_hist, w, np.float64)
    oe /= np.linalg.norm(oe)
    os_ /= np.linalg.norm(os_)
    errs = (helpers.rel_l2(tr.cpu().numpy(), o_tr), helpers.rel_l2(ge.cpu().numpy(), oe),
            helpers.rel_l2(gs.cpu().numpy(), os_))
    print("config1 (nt 1000) vs FP64 oracle: traces %.3g, g_eps %.3g, g_sig %.3g" % errs)
    assert all(np.isfinite(e) for e in errs) and max(errs) <= TOL_FP64


@pytest.mark.parametrize("tuning", [None, BAND])
def test_config2_sample_vs_reference_kernels(fg, dev, refdrv, tuning):
    errs = _vs_reference(fg, refdrv, fg.workloads.config2(shots=64, nt=1000), dev, tuning=tuning)
    assert max(errs) <= TOL_REF


def test_edge_shapes_checked_build():
    env = dict(os.environ, FASTGPR_CHECKED="1")
    r = subprocess.run([sys.executable, os.path.join(HERE, "checked_edge_shapes.py")], env=env, capture_output=True,
                       text=True, timeout=1200)
    print(r.stdout[-2000:], r.stderr[-4000:])
    assert r.returncode == 0 and r.stdout.strip().splitlines()[-1].startswith("ok ")


def test_l1_adjoint_vs_oracle(fg, orc, dev):
    """fg_adjoint_reference_l1 injects scale * sign(traces - observed) formed in
    the adjoint step; the oracle gets that residual formed on the host."""
    for wl in (fg.workloads.small(), fg.workloads.small(seed=3, shots=2, nt=150, nx=40, ny=56, pml=5, nrx=6)):
        prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
        solve = fg.Solve(dev, setup, tv=False)
        er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
        traces, hist = solve.forward(er, se, mr)
        rng = np.random.default_rng(9)
        obs = traces + torch.tensor(rng.standard_normal(traces.shape).astype(np.float32), device=dev) * \
            traces.abs().max()
        obs[:, :5] = traces[:, :5]   # some exact zeros of the residual (sign 0)
        scale = float(np.float32(1.0 / traces.numel()))
        ge = torch.empty((setup.nx, setup.ny), device=dev)
        gs = torch.empty_like(ge)
        solve.plan.adjoint_reference_l1(*solve.materials(er, se, mr), hist, traces, obs, scale, ge, gs,
                                        normalize=False)
        d = traces.cpu().numpy() - obs.cpu().numpy()
        resid = (np.sign(d) * np.float32(scale)).astype(np.float32)
        o_tr, o_hist = orc.forward(prob, np.float32)
        oe, os_ = orc.adjoint_reference(prob, o_hist, resid, np.float64)
        assert helpers.rel_l2(ge.cpu().numpy(), oe) < 1e-6
        assert helpers.rel_l2(gs.cpu().numpy(), os_) < 1e-6
