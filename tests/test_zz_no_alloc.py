"""fg_forward_static: the forward solve for callers that cannot allocate
device memory.

cudaMalloc and cudaFree may synchronise the whole device, and some host
applications give all device memory to their own pool up front; a caller in
either position allocates only its inputs and outputs and lets this entry
point place the solver's scratch in the library's fixed device array
(FG_STATIC_SCRATCH_BYTES).  These tests call it through the C ABI and compare
it with fg_forward, the entry point that uses a caller-allocated workspace.

The file name makes pytest collect it last, so a run that stops at the first
failure has run every other test before this one.
"""
import ctypes
import importlib

import numpy as np
import pytest
import torch

import helpers

PKG = "fast-gpr-fwi_b200"


def _problem(nx, ny, shots, nt, th):
    """An fg_problem with one source and one receiver per shot (host tables)."""
    nat = helpers.native_mod()
    src = np.tile(np.array([[[nx // 3, ny // 3, 0]]], np.int32), (shots, 1, 1))
    rx = np.tile(np.array([[[nx // 2, ny // 2, 0]]], np.int32), (shots, 1, 1))
    srcw = np.ones((1, nt), np.float32)
    pml = np.full((8, th), 0.5, np.float32)
    prob = nat.FgProblem()
    prob.nx, prob.ny, prob.shots, prob.nt, prob.th = nx, ny, shots, nt, th
    prob.dx, prob.dt = 0.025, 5e-11
    prob.nsrc, prob.nrx = 1, 1
    prob.src = src.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    prob.rx = rx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    prob.srcw = srcw.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    prob.pml = pml.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    return prob, (src, rx, srcw, pml)


def test_forward_static_rejects_plans_beyond_the_static_scratch(fg):
    """The size check happens on the host, before any device work."""
    nat = helpers.native_mod()
    L = nat.lib()
    prob, keep = _problem(440, 340, 64, 10, 20)
    h = ctypes.c_void_p()
    assert L.fg_plan_create(ctypes.byref(prob), None, ctypes.byref(h)) == nat.FG_OK
    try:
        assert L.fg_plan_workspace_bytes(h) > 32 * 1024 * 1024
        rc = L.fg_forward_static(h, None, None, None, None, None, None)
        assert rc == nat.FG_ERR_WORKSPACE
        assert b"static" in L.fg_last_error()
    finally:
        L.fg_plan_destroy(h)


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", [None, {"kernel": 0, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 4},
                                    {"kernel": 2, "lanes": 1, "cells_per_thread": 4, "rows_per_tile": 8}])
def test_forward_static_matches_forward(fg, tuning):
    """Two calls in a row through the C ABI give the traces and history of
    fg_forward bit for bit (the forward tests' tolerance), for the default
    launch shape, the tile pipeline (whose tensor maps are pointed at the
    array and back) and the band pipeline."""
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    dev = torch.device("cuda:0")
    nat = helpers.native_mod()
    L = nat.lib()
    wl = fg.workloads.small(shots=3, nt=90)
    setup = helpers.setup_for(wl, dev)
    solve = fg.Solve(dev, setup, tv=False, tuning=tuning)
    assert L.fg_plan_workspace_bytes(solve.plan.handle) <= 32 * 1024 * 1024
    er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
    want_tr, want_hist = solve.forward(er, se, mr)
    torch.cuda.synchronize()
    stream = nat.stream_handle(dev)
    for call in range(2):
        tr = torch.full_like(want_tr, float("nan"))
        hist = torch.full_like(want_hist, float("nan"))
        nat.check(L.fg_forward_static(solve.plan.handle, er.data_ptr(), se.data_ptr(), mr.data_ptr(),
                                      tr.data_ptr(), hist.data_ptr(), stream))
        torch.cuda.synchronize()
        assert torch.equal(tr, want_tr), "call %d: traces differ from fg_forward" % call
        assert torch.equal(hist, want_hist), "call %d: history differs from fg_forward" % call
    # the plan's own workspace binding is untouched: fg_forward still works on it
    tr2, hist2 = solve.forward(er, se, mr)
    torch.cuda.synchronize()
    assert torch.equal(tr2, want_tr) and torch.equal(hist2, want_hist)


@pytest.mark.gpu
def test_forward_static_two_plans_in_turn(fg):
    """Plans that take turns re-upload their tables into the shared array:
    A, B, A again each match their own fg_forward."""
    dev = torch.device("cuda:0")
    nat = helpers.native_mod()
    L = nat.lib()
    runs = []
    for wl in (fg.workloads.small(shots=3, nt=80), fg.workloads.small(seed=3, shots=2, nt=60, nx=40, ny=56, pml=5)):
        solve = fg.Solve(dev, helpers.setup_for(wl, dev), tv=False)
        er, se, mr = (torch.tensor(a, device=dev) for a in (wl.er, wl.se, wl.mr))
        want = solve.forward(er, se, mr)
        runs.append((solve, (er, se, mr), want))
    torch.cuda.synchronize()
    stream = nat.stream_handle(dev)
    for k in (0, 1, 0):
        solve, (er, se, mr), (want_tr, want_hist) = runs[k]
        tr = torch.full_like(want_tr, float("nan"))
        hist = torch.full_like(want_hist, float("nan"))
        nat.check(L.fg_forward_static(solve.plan.handle, er.data_ptr(), se.data_ptr(), mr.data_ptr(),
                                      tr.data_ptr(), hist.data_ptr(), stream))
        torch.cuda.synchronize()
        assert torch.equal(tr, want_tr) and torch.equal(hist, want_hist), "plan %d" % k
