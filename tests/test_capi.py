"""The C-ABI library loads and exports every entry point include/fastgpr.h declares."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "fastgpr.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fg_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "fg_forward" in syms and "fg_adjoint_reference" in syms and "fg_coefficients" in syms


def test_library_exports_every_declared_symbol(fg):
    nat = __import__("importlib").import_module("fast-gpr-fwi_b200._native")
    for checked in (False, True):
        path = nat.library_path(checked)
        assert os.path.exists(path), "library not built: %s" % path
        lib = ctypes.CDLL(path)
        for s in declared_symbols():
            assert hasattr(lib, s), "%s does not export %s" % (os.path.basename(path), s)
    assert set(declared_symbols()) == set(nat.EXPORTS)


def test_plan_validation_without_gpu(fg):
    """Host-side argument checks run before any device work."""
    import numpy as np
    import pytest
    nat = __import__("importlib").import_module("fast-gpr-fwi_b200._native")
    L = nat.lib()
    src = np.zeros((1, 1, 3), np.int32)
    rx = np.array([[[5, 5, 0]]], np.int32)
    srcw = np.ones((1, 4), np.float32)
    prob = nat.FgProblem()
    prob.nx, prob.ny, prob.shots, prob.nt, prob.th = 8, 8, 1, 4, 0
    prob.dx, prob.dt = 0.1, 1e-10
    prob.nsrc, prob.nrx = 1, 1
    prob.src = src.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    prob.rx = rx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    prob.srcw = srcw.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    h = ctypes.c_void_p()
    assert L.fg_plan_create(ctypes.byref(prob), None, ctypes.byref(h)) == nat.FG_OK
    assert L.fg_plan_workspace_bytes(h) > 0
    L.fg_plan_destroy(h)
    rx[0, 0, 0] = 9   # beyond the i == nx frame
    assert L.fg_plan_create(ctypes.byref(prob), None, ctypes.byref(h)) == nat.FG_ERR_INVALID
    assert b"receiver" in L.fg_last_error()
    rx[0, 0, 0] = 8   # on the frame: inert, accepted
    assert L.fg_plan_create(ctypes.byref(prob), None, ctypes.byref(h)) == nat.FG_OK
    L.fg_plan_destroy(h)
    prob.th = 5       # 2*th > nx
    assert L.fg_plan_create(ctypes.byref(prob), None, ctypes.byref(h)) == nat.FG_ERR_INVALID
    with pytest.raises(nat.FastGprError):
        nat.check(nat.FG_ERR_INVALID)


def test_tv_workspace_size_without_gpu(fg):
    from importlib import import_module
    nat = import_module("fast-gpr-fwi_b200._native")
    L = nat.lib()
    assert L.fg_tv_workspace_bytes(440, 340) >= 7 * 442 * 342 * 4
    assert L.fg_tv_workspace_bytes(0, 5) == -1


def test_checkpoint_sizes_and_adjoint_tuning_without_gpu(fg):
    """Checkpoint buffer sizes and adjoint launch-shape validation are host-side."""
    import numpy as np
    nat = __import__("importlib").import_module("fast-gpr-fwi_b200._native")
    L = nat.lib()
    src = np.array([[[3, 3, 0]]], np.int32)
    rx = np.array([[[5, 5, 0]]], np.int32)
    nt = 50
    srcw = np.ones((1, nt), np.float32)
    prob = nat.FgProblem()
    prob.nx, prob.ny, prob.shots, prob.nt, prob.th = 16, 12, 1, nt, 0
    prob.dx, prob.dt = 0.1, 1e-10
    prob.nsrc, prob.nrx = 1, 1
    prob.src = src.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    prob.rx = rx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    prob.srcw = srcw.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    h = ctypes.c_void_p()
    assert L.fg_plan_create(ctypes.byref(prob), None, ctypes.byref(h)) == nat.FG_OK
    one = L.fg_plan_checkpoint_bytes(h, 49)          # two segments: one checkpoint
    assert one > 0
    assert L.fg_plan_checkpoint_bytes(h, 50) == 0     # one segment: the initial state is zero
    assert L.fg_plan_checkpoint_bytes(h, 1000) == 0
    assert L.fg_plan_checkpoint_bytes(h, 10) == 4 * one
    assert L.fg_plan_checkpoint_bytes(h, 1) == (nt - 1) * one
    assert L.fg_plan_checkpoint_bytes(h, 0) == -1
    L.fg_plan_destroy(h)
    bad = nat.FgTuning(*([0] * 6 + [4, 0, 0, 0]))     # adj_kernel 4 does not exist
    assert L.fg_plan_create(ctypes.byref(prob), ctypes.byref(bad), ctypes.byref(h)) == nat.FG_ERR_INVALID
    assert b"adj_kernel" in L.fg_last_error()
    ok = nat.FgTuning(*([0] * 6 + [2, 3, 2, 0]))      # lane-march adjoint
    assert L.fg_plan_create(ctypes.byref(prob), ctypes.byref(ok), ctypes.byref(h)) == nat.FG_OK
    L.fg_plan_destroy(h)


def _shape_of(nat, nx, ny, shots, tuning=None, th=20):
    """Launch shapes of a plan (host-side) for an nx x ny grid with `shots` shots."""
    import numpy as np
    src = np.zeros((shots, 1, 3), np.int32)
    src[:, 0, 0] = th + 2
    src[:, 0, 1] = np.arange(shots) % (ny - 2 * th - 4) + th + 2
    rx = np.zeros((shots, 1, 3), np.int32)
    rx[:, 0, 0] = nx - th - 3
    rx[:, 0, 1] = ny // 2
    p = nat.Plan(nx, ny, shots, 8, th, 0.025, 4e-11, src, rx, np.ones((1, 8), np.float32),
                 np.zeros(8 * th, np.float32), "cuda:0", tuning=tuning, bind=False)
    return p.shape()


def test_default_launch_shapes_by_step_size(fg):
    """The size-dependent defaults (host-side, no GPU): interior split from
    12,000 cells x shot groups; the adjoint's slab kernel at 2 / 1 blocks per
    SM below 5e4 / 1.2e5; forward tiles of 2 rows below 1.2e5; the adjoint's
    8 cells per thread from 2e5; column lanes below 8 shots; no split in a
    persistent plan."""
    nat = __import__("importlib").import_module("fast-gpr-fwi_b200._native")
    tiny = _shape_of(nat, 100, 80, 8)                      # 8,000 cells x 1 group
    assert tiny["forward"]["interior_split"] == 0 and tiny["adjoint"]["interior_split"] == 0
    assert tiny["forward"]["rows_per_tile"] == 2 and tiny["adjoint"]["rows_per_tile"] == 4
    small = _shape_of(nat, 140, 100, 16)                   # 14,000
    assert small["forward"]["interior_split"] == 1 and small["adjoint"]["interior_split"] == 1
    assert small["forward"]["slab_blocks_per_sm"] == 2 and small["adjoint"]["slab_blocks_per_sm"] == 2
    assert small["forward"]["rows_per_tile"] == 2 and small["adjoint"]["cells_per_thread"] == 4
    mid = _shape_of(nat, 296, 296, 32)                     # 87,616
    assert mid["adjoint"]["slab_blocks_per_sm"] == 1 and mid["forward"]["rows_per_tile"] == 2
    one_group = _shape_of(nat, 440, 340, 32)               # 149,600
    assert one_group["adjoint"]["slab_blocks_per_sm"] == 0 and one_group["forward"]["rows_per_tile"] == 4
    assert one_group["adjoint"]["cells_per_thread"] == 4
    bench = _shape_of(nat, 440, 340, 64)                   # 299,200: the benchmark grid
    assert bench["forward"] == dict(kernel=1, lanes=1, cells_per_thread=4, rows_per_tile=4, warps_per_block=4,
                                    stages=0, interior_split=1, slab_blocks_per_sm=2, persistent=0)
    assert bench["adjoint"] == dict(kernel=1, lanes=1, cells_per_thread=8, rows_per_tile=4, warps_per_block=4,
                                    stages=0, interior_split=1, slab_blocks_per_sm=0, persistent=0)
    pers = _shape_of(nat, 140, 100, 16, tuning={"lanes": 1, "persistent": 1})
    assert pers["forward"]["persistent"] == 1 and pers["forward"]["interior_split"] == 0
    assert pers["forward"]["rows_per_tile"] == 4
    col = _shape_of(nat, 440, 340, 3)
    assert col["forward"]["lanes"] == 2 and col["forward"]["kernel"] == 0 and col["forward"]["interior_split"] == 0
    forced = _shape_of(nat, 440, 340, 64, tuning={"interior": -1, "slab": -1})
    assert forced["forward"]["interior_split"] == 0 and forced["adjoint"]["interior_split"] == 0
