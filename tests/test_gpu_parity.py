"""GPU parity: the CUDA path against the CPU oracle (bit-exact forward) and
against the reference's own CUDA kernels (oracle/_ref, driven by
oracle/ref_driver.py): traces and reference-mode gradients within 1e-5
relative L2, FP32 gradient error against the FP64 oracle stated and bounded
by 1e-4."""
import importlib

import numpy as np
import pytest
import torch

import helpers

pytestmark = pytest.mark.gpu

TOL_REF = 1e-5     # relative L2 vs the reference kernels (traces, gradients)
TOL_FP64 = 1e-4    # relative L2 of the FP32 gradient vs the FP64 oracle


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


def _cases(fg):
    return [fg.workloads.small(), fg.workloads.small(seed=3, shots=2, nt=150, nx=40, ny=56, pml=5, nrx=6),
            fg.workloads.config0()]


def _run_package(fg, wl, dev, w, tuning=None, tv=False):
    er = torch.tensor(wl.er[:, :, None], device=dev, requires_grad=True)
    se = torch.tensor(wl.se[:, :, None], device=dev, requires_grad=True)
    traces, dt = fg.compute(**wl.kwargs(dev, er=er, se=se, tv=tv, tuning=tuning))
    (traces * w).sum().backward()
    torch.cuda.synchronize()
    return traces.detach(), er.grad[:, :, 0].detach(), se.grad[:, :, 0].detach()


def _run_reference(refdrv, wl, dev, w):
    kw = wl.kwargs(dev)
    er = torch.clamp(kw["er"], min=1)
    se = torch.clamp(kw["se"], min=0)
    G = refdrv.setup(dev, kw["dx"], kw["ny"], kw["nx"], 1, kw["time_windows"], kw["source_location"],
                     kw["source_step"], kw["receiver_location"], kw["receiver_step"], kw["pmlthick"],
                     kw["source_apmlitudes"], kw["step"], er, se, kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"],
                     kw["Fixedreceiver"])
    rxs, hist = refdrv.forward(G)
    ge, gs = refdrv.backward(G, er, se, kw["mr"], hist, w)
    return G, rxs[:, 2].contiguous(), ge[:, :, 0], gs[:, :, 0]


def test_coefficients_bit_exact_vs_reference(fg, dev, refdrv):
    nat = helpers.native_mod()
    for wl in _cases(fg):
        kw = wl.kwargs(dev)
        er = torch.clamp(kw["er"], min=1)
        se = torch.clamp(kw["se"], min=0)
        G = refdrv.setup(dev, kw["dx"], kw["ny"], kw["nx"], 1, kw["time_windows"], kw["source_location"],
                         kw["source_step"], kw["receiver_location"], kw["receiver_step"], kw["pmlthick"],
                         kw["source_apmlitudes"], kw["step"], er, se, kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"],
                         kw["Fixedreceiver"])
        e32 = er[:, :, 0].float().contiguous()
        s32 = se[:, :, 0].float().contiguous()
        m32 = kw["mr"][:, :, 0].float().contiguous()
        mine = nat.coefficients(e32, s32, m32, float(np.float32(G.dt)), float(np.float32(G.dx)), False)
        nx, ny = wl.nx, wl.ny
        ref = G.coef_single   # uE0 uE1 uE4 uH0 uH1 uH4, (nx+1, ny+1, 2)
        for k, r in ((0, 0), (1, 1), (2, 2), (3, 4), (4, 5)):
            a = mine[k, :nx, :ny].cpu().numpy()
            b = ref[r][:nx, :ny, 0].cpu().numpy()
            assert np.array_equal(a, b), "coefficient plane %d differs (%d cells)" % (k, int((a != b).sum()))
        H = refdrv.Grid()
        for k in ("step", "device", "dx", "dy", "dz", "nx", "ny", "nz", "dt"):
            setattr(H, k, getattr(G, k))
        refdrv._coefficients(H, er, se, kw["mr"], adjoint=True)
        mine_a = nat.coefficients(e32, s32, m32, float(np.float32(G.dt)), float(np.float32(G.dx)), True)
        a = mine_a[0, :nx, :ny].cpu().numpy()
        b = H.coef_single[0][:nx, :ny, 0].cpu().numpy()
        mism = int((a != b).sum())
        ulp = np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64)).max()
        assert ulp <= 1, "adjoint uE0 differs by %d ulp in %d cells" % (ulp, mism)


def test_setup_matches_reference(fg, dev, refdrv):
    for wl in _cases(fg):
        kw = wl.kwargs(dev)
        er = torch.clamp(kw["er"], min=1)
        se = torch.clamp(kw["se"], min=0)
        G = refdrv.setup(dev, kw["dx"], kw["ny"], kw["nx"], 1, kw["time_windows"], kw["source_location"],
                         kw["source_step"], kw["receiver_location"], kw["receiver_step"], kw["pmlthick"],
                         kw["source_apmlitudes"], kw["step"], er, se, kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"],
                         kw["Fixedreceiver"])
        s = helpers.setup_for(wl, dev)
        assert s.nt == G.iterations
        assert torch.equal(s.src.cpu(), G.source[:wl.shots].cpu())
        assert torch.equal(s.rx.cpu(), G.receiver[:wl.shots].cpu())
        p = G.pmls[0]
        ref_pml = np.concatenate([t.cpu().numpy() for t in (p.ERA, p.ERB, p.ERE, p.ERF, p.HRA, p.HRB, p.HRE, p.HRF)])
        assert np.array_equal(s.profile.packed(), ref_pml)
        d = np.float32(wl.dx)
        w = G.waveform.cpu().numpy()
        np.testing.assert_array_equal(s.srcw[0], (w * d) / ((d * d) * d))


TUNINGS = [
    None,
    # tensor-map tiles
    {"lanes": 1, "cells_per_thread": 4, "rows_per_tile": 2},
    {"lanes": 1, "cells_per_thread": 8, "rows_per_tile": 8, "stages": 2},
    {"lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "stages": 4},
    {"lanes": 2, "cells_per_thread": 2, "rows_per_tile": 8},
    {"lanes": 2, "cells_per_thread": 4, "rows_per_tile": 2},
    {"lanes": 1, "cells_per_thread": 4, "rows_per_tile": 16, "warps_per_block": 4},
    {"lanes": 1, "cells_per_thread": 4, "rows_per_tile": 8, "warps_per_block": 1, "stages": 2},
    {"lanes": 2, "cells_per_thread": 2, "rows_per_tile": 16, "warps_per_block": 8},
    # lane march
    {"kernel": 1, "lanes": 1, "cells_per_thread": 2, "rows_per_tile": 3},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 8, "rows_per_tile": 7, "warps_per_block": 1},
    {"kernel": 1, "lanes": 2, "cells_per_thread": 4, "rows_per_tile": 1},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 9, "stages": 2},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 8, "rows_per_tile": 16, "warps_per_block": 2, "stages": 4},
    {"kernel": 1, "lanes": 2, "cells_per_thread": 2, "rows_per_tile": 6, "stages": 3},
    # the whole time loop in one persistent launch
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "persistent": 1},
    {"kernel": 1, "lanes": 2, "cells_per_thread": 2, "rows_per_tile": 5, "persistent": 1},
    {"kernel": 1, "lanes": 2, "cells_per_thread": 8, "rows_per_tile": 2, "persistent": 1},
    # the interior split forced on small grids (general kernel at 1 and 2 blocks per SM)
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "interior": 2},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 2, "rows_per_tile": 3, "interior": 1, "prefetch": 2},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 8, "rows_per_tile": 2, "interior": 2, "adj_kernel": 2,
     "adj_cells_per_thread": 4},
    # the slab kernels (x-slab and y-slab tiles) for the forward and the adjoint, forced on small grids
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "interior": 2, "slab": 1},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 8, "rows_per_tile": 3, "interior": 1, "slab": 3},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 2, "rows_per_tile": 2, "interior": 2, "slab": 2, "adj_kernel": 2,
     "adj_cells_per_thread": 4},
    # shot pairs (two shots per lane)
    {"kernel": 1, "lanes": 3, "cells_per_thread": 2, "rows_per_tile": 4},
    {"kernel": 1, "lanes": 3, "cells_per_thread": 4, "rows_per_tile": 5},
    # forward and adjoint on different launch shapes
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "adj_kernel": 1, "adj_rows_per_tile": 8,
     "adj_warps_per_block": 4, "adj_stages": 2},
    {"kernel": 0, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 8, "adj_kernel": 2, "adj_rows_per_tile": 3},
    # the adjoint on its own cells per thread
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "adj_kernel": 2, "adj_rows_per_tile": 4,
     "adj_cells_per_thread": 8},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "adj_kernel": 1, "adj_rows_per_tile": 4,
     "adj_warps_per_block": 4, "adj_stages": 2, "adj_cells_per_thread": 8},
    {"kernel": 1, "lanes": 2, "cells_per_thread": 2, "rows_per_tile": 4, "adj_kernel": 2, "adj_cells_per_thread": 4},
    # band pipeline (the adjoint follows the forward's shape)
    {"kernel": 2, "lanes": 1, "cells_per_thread": 4, "warps_per_block": 4, "rows_per_tile": 7, "stages": 3},
    {"kernel": 2, "lanes": 1, "cells_per_thread": 2, "warps_per_block": 4, "rows_per_tile": 16},
    {"kernel": 2, "lanes": 1, "cells_per_thread": 4, "warps_per_block": 2, "rows_per_tile": 1, "stages": 2},
    {"kernel": 2, "lanes": 1, "cells_per_thread": 2, "warps_per_block": 8, "rows_per_tile": 64, "stages": 8},
    # band-pipeline adjoint behind other forwards
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "adj_kernel": 3, "adj_rows_per_tile": 9,
     "adj_cells_per_thread": 4, "adj_warps_per_block": 4, "adj_stages": 4},
    {"lanes": 1, "adj_kernel": 3, "adj_cells_per_thread": 2, "adj_warps_per_block": 8},
]


@pytest.mark.parametrize("tuning", TUNINGS)
def test_forward_bit_exact_vs_oracle(fg, orc, dev, tuning):
    for wl in _cases(fg)[:2]:
        prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
        solve = fg.Solve(dev, setup, tuning=tuning, tv=False)
        traces, hist = solve.forward(torch.tensor(wl.er, device=dev), torch.tensor(wl.se, device=dev),
                                     torch.tensor(wl.mr, device=dev))
        o_tr, o_hist = orc.forward(prob, np.float32)
        np.testing.assert_array_equal(traces.cpu().numpy(), o_tr)
        np.testing.assert_array_equal(solve.plan.hist_view(hist).cpu().numpy(), o_hist)


@pytest.mark.parametrize("tuning", TUNINGS)
def test_adjoint_vs_oracle(fg, orc, dev, tuning):
    for wl in _cases(fg)[:2]:
        prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
        solve = fg.Solve(dev, setup, tv=False, tuning=tuning)
        er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
        traces, hist = solve.forward(er, se, mr)
        rng = np.random.default_rng(5)
        resid = rng.standard_normal(traces.shape).astype(np.float32)
        ge, gs = solve.gradient(er, se, mr, hist, torch.tensor(resid, device=dev), normalize=False)
        o_tr, o_hist = orc.forward(prob, np.float32)
        oe, os_ = orc.adjoint_reference(prob, o_hist, resid, np.float64)
        assert helpers.rel_l2(ge.cpu().numpy(), oe) < 1e-6
        assert helpers.rel_l2(gs.cpu().numpy(), os_) < 1e-6


def test_traces_and_gradient_vs_reference_kernels(fg, dev, refdrv):
    for wl in _cases(fg):
        rng = np.random.default_rng(17)
        w = torch.tensor(rng.standard_normal((wl.shots, wl.nt, wl.nrx)).astype(np.float32), device=dev)
        tr, ge, gs = _run_package(fg, wl, dev, w)
        G, rtr, rge, rgs = _run_reference(refdrv, wl, dev, w)
        e_tr = helpers.rel_l2(tr.cpu().numpy(), rtr.cpu().numpy())
        e_ge = helpers.rel_l2(ge.cpu().numpy(), rge.cpu().numpy())
        e_gs = helpers.rel_l2(gs.cpu().numpy(), rgs.cpu().numpy())
        print("%s vs reference kernels: traces %.3g, g_eps %.3g, g_sig %.3g" % (wl.name, e_tr, e_ge, e_gs))
        assert e_tr <= TOL_REF and e_ge <= TOL_REF and e_gs <= TOL_REF


def test_gradient_error_vs_fp64_oracle(fg, orc, dev):
    for wl in _cases(fg):
        rng = np.random.default_rng(23)
        w = rng.standard_normal((wl.shots, wl.nt, wl.nrx)).astype(np.float32)
        tr, ge, gs = _run_package(fg, wl, dev, torch.tensor(w, device=dev))
        prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
        f64 = orc.coefficients_fp64(np.maximum(wl.er, 1), np.maximum(wl.se, 0), wl.mr, setup.dt32, setup.dx)
        p64 = prob.cast(np.float64)
        for k, v in f64.items():
            setattr(p64, k, v)
        er_avg = float(np.mean(np.maximum(wl.er, 1)[0, :].astype(np.float64)))
        p64.pml = orc.cpml_fp64(setup.th, setup.dx, er_avg, 1.0, setup.dt32)
        p64.srcw = np.zeros_like(prob.srcw, dtype=np.float64)
        p64.srcw[0] = orc.ricker_fp64(setup.nt, setup.dt32, (wl.nt - 1.5) * wl.dt, 1.0, wl.freq, setup.dx)
        o_tr, o_hist = orc.forward(p64, np.float64)
        oe, os_ = orc.adjoint_reference(p64, o_hist, w, np.float64)
        oe /= np.linalg.norm(oe)
        os_ /= np.linalg.norm(os_)
        e_tr = helpers.rel_l2(tr.cpu().numpy(), o_tr)
        e_ge = helpers.rel_l2(ge.cpu().numpy(), oe)
        e_gs = helpers.rel_l2(gs.cpu().numpy(), os_)
        print("%s vs FP64 oracle: traces %.3g, g_eps %.3g, g_sig %.3g" % (wl.name, e_tr, e_ge, e_gs))
        assert e_ge <= TOL_FP64 and e_gs <= TOL_FP64


def test_tiling_invariance(fg, dev):
    wl = fg.workloads.small(shots=5, nt=100)
    w = torch.ones((wl.shots, wl.nt, wl.nrx), device=dev)
    base = _run_package(fg, wl, dev, w)
    for tuning in TUNINGS[1:]:
        got = _run_package(fg, wl, dev, w, tuning=tuning)
        assert torch.equal(got[0], base[0])
        for a, b in zip(got[1:], base[1:]):
            assert helpers.rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("lanes", [1, 2])
def test_shot_alone_equals_shot_in_batch(fg, dev, lanes):
    wl = fg.workloads.small(shots=4, nt=100)
    w = torch.ones((wl.shots, wl.nt, wl.nrx), device=dev)
    tr, _, _ = _run_package(fg, wl, dev, w, tuning={"lanes": lanes})
    setup = helpers.setup_for(wl, dev)
    for s in range(wl.shots):
        er = torch.tensor(wl.er[:, :, None], device=dev)
        se = torch.tensor(wl.se[:, :, None], device=dev)
        kw = wl.kwargs(dev, er=er, se=se, tv=False, step=1, customsource=setup.src[s:s + 1].clone(),
                       customreceiver=setup.rx[s:s + 1].clone())
        tr1, _ = fg.compute(**kw)
        assert torch.equal(tr1[0], tr[s])


@pytest.mark.parametrize("shots,tuning", [
    (37, None),
    (37, {"lanes": 3, "kernel": 1, "cells_per_thread": 2}),
    (70, {"lanes": 3, "kernel": 1, "cells_per_thread": 4, "rows_per_tile": 3}),
])
def test_two_shot_groups_vs_oracle(fg, orc, dev, shots, tuning):
    """More shots than one group holds (32 shot lanes, 64 shot pairs): two
    shot groups, the second padded; or one padded group of pairs."""
    wl = fg.workloads.small(shots=shots, nt=70, fixed=True, nx=64)
    wl.source_step = [0.03, 0.01, 0.0]
    prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
    solve = fg.Solve(dev, setup, tv=False, tuning=tuning)
    er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
    traces, hist = solve.forward(er, se, mr)
    o_tr, o_hist = orc.forward(prob, np.float32)
    np.testing.assert_array_equal(traces.cpu().numpy(), o_tr)
    np.testing.assert_array_equal(solve.plan.hist_view(hist).cpu().numpy(), o_hist)
    rng = np.random.default_rng(8)
    resid = rng.standard_normal(traces.shape).astype(np.float32)
    ge, gs = solve.gradient(er, se, mr, hist, torch.tensor(resid, device=dev), normalize=False)
    oe, os_ = orc.adjoint_reference(prob, o_hist, resid, np.float64)
    assert helpers.rel_l2(ge.cpu().numpy(), oe) < 1e-6
    assert helpers.rel_l2(gs.cpu().numpy(), os_) < 1e-6


@pytest.mark.parametrize("scale,dx", [(1e13, 0.05), (1e-20, 0.05), (1.0, 0.03)])
@pytest.mark.parametrize("tuning", [
    None,
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4},
    {"kernel": 1, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4, "adj_kernel": 1, "adj_rows_per_tile": 8,
     "adj_warps_per_block": 4, "adj_stages": 2},
])
def test_division_ranges_vs_oracle(fg, orc, dev, scale, dx, tuning):
    """Field values that take each branch of the CPML rows' division by the
    cell size: derivatives of 2^31 and above (amplitude 1e13: the per-division
    path of the shot-lane rows), fields around 1e-18 with tens of thousands of
    subnormal values at the wavefront (the scaled step, whose double rounding
    the bind-time check rules out for dx = 0.05), and dx = 0.03, whose scaled
    step fails that check (subnormal quotients round differently), so its
    rows divide per cell throughout."""
    wl = fg.workloads.small(shots=3, nt=120, dx=dx, nx=64)
    prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
    prob.srcw = setup.srcw = np.ascontiguousarray(setup.srcw * np.float32(scale), dtype=np.float32)
    solve = fg.Solve(dev, setup, tv=False, tuning=tuning)
    er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
    traces, hist = solve.forward(er, se, mr)
    o_tr, o_hist = orc.forward(prob, np.float32)
    assert np.isfinite(o_tr).all() and np.abs(o_tr).max() > 0
    np.testing.assert_array_equal(traces.cpu().numpy(), o_tr)
    np.testing.assert_array_equal(solve.plan.hist_view(hist).cpu().numpy(), o_hist)
    # the residual scales up with a large source, never down, so that the
    # gradients stay inside float32's normal range
    rng = np.random.default_rng(9)
    resid = (rng.standard_normal(traces.shape) * max(scale, 1.0)).astype(np.float32)
    ge, gs = solve.gradient(er, se, mr, hist, torch.tensor(resid, device=dev), normalize=False)
    oe, os_ = orc.adjoint_reference(prob, o_hist, resid, np.float64)
    assert helpers.rel_l2(ge.cpu().numpy(), oe) < 1e-6
    assert helpers.rel_l2(gs.cpu().numpy(), os_) < 1e-6


@pytest.mark.parametrize("grid", [(130, 100, 9), (200, 170, 33)])
def test_default_shapes_on_split_sized_grids_vs_oracle(fg, orc, dev, grid):
    """The default launch shapes of shot-lane steps of at least 12,000 cells x
    shot groups (interior split, the adjoint's slab kernel at 2 / 1 blocks
    per SM, 2-row forward tiles): traces and history bit-exact against the
    oracle, gradients within 1e-6."""
    nx, ny, shots = grid
    wl = fg.workloads.small(seed=nx + ny, nx=nx, ny=ny, shots=shots, nt=40, pml=10, nrx=7, fixed=True)
    wl.source_step = [0.05, 0.03, 0.0]
    prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
    solve = fg.Solve(dev, setup, tv=False)
    shape = solve.plan.shape()
    assert shape["forward"]["interior_split"] == 1 and shape["forward"]["rows_per_tile"] == 2
    assert shape["adjoint"]["interior_split"] == 1 and shape["adjoint"]["slab_blocks_per_sm"] in (1, 2)
    er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
    traces, hist = solve.forward(er, se, mr)
    o_tr, o_hist = orc.forward(prob, np.float32)
    np.testing.assert_array_equal(traces.cpu().numpy(), o_tr)
    np.testing.assert_array_equal(solve.plan.hist_view(hist).cpu().numpy(), o_hist)
    rng = np.random.default_rng(8)
    resid = rng.standard_normal(traces.shape).astype(np.float32)
    ge, gs = solve.gradient(er, se, mr, hist, torch.tensor(resid, device=dev), normalize=False)
    oe, os_ = orc.adjoint_reference(prob, o_hist, resid, np.float64)
    assert helpers.rel_l2(ge.cpu().numpy(), oe) < 1e-6
    assert helpers.rel_l2(gs.cpu().numpy(), os_) < 1e-6
