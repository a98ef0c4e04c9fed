"""Edge-shape sweep for the bounds-checked build (run by
tests/test_gpu_configs.py in a process of its own with FASTGPR_CHECKED=1, so
that libfastgpr_checked.so is the library loaded).

Every grid nx, ny in {17, 33, 65} with CPML thickness 0, 1 or 8, for each
kernel family, runs a forward + reference-mode adjoint; each call is
followed by fg_plan_check, which raises if a kernel recorded an out-of-range
access or a wait that gave up.  Forward traces must equal the oracle's bit
for bit and the gradients must match its FP64 imaging sums within 1e-6.
Prints "ok <cases>" at the end."""
import itertools
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import importlib  # noqa: E402

import helpers  # noqa: E402
from oracle import oracle as orc  # noqa: E402

TUNINGS = [
    None,
    {"lanes": 1, "kernel": 1, "cells_per_thread": 4, "rows_per_tile": 4, "adj_kernel": 2, "adj_cells_per_thread": 8},
    {"lanes": 1, "kernel": 2, "cells_per_thread": 4, "warps_per_block": 4, "rows_per_tile": 8, "stages": 4},
    {"lanes": 1, "kernel": 0, "cells_per_thread": 4, "rows_per_tile": 4},
    {"lanes": 2},
    # the persistent launch; the interior split forced (few or no interior tiles)
    {"lanes": 1, "kernel": 1, "cells_per_thread": 4, "rows_per_tile": 4, "persistent": 1},
    {"lanes": 1, "kernel": 1, "cells_per_thread": 4, "rows_per_tile": 2, "interior": 2},
    {"lanes": 2, "kernel": 1, "cells_per_thread": 4, "persistent": 1},
    # the slab kernels of both solves, the frame rows and columns included
    {"lanes": 1, "kernel": 1, "cells_per_thread": 4, "rows_per_tile": 3, "interior": 2, "slab": 2},
]


def main():
    fg = importlib.import_module("fast-gpr-fwi_b200")
    nat = helpers.native_mod()
    assert nat.checked_build(), "run with FASTGPR_CHECKED=1"
    dev = torch.device("cuda:0")
    n = 0
    for nx, ny, pml in itertools.product((17, 33, 65), (17, 33, 65), (0, 1, 8)):
        wl = helpers.edge_workload(fg, nx, ny, pml)
        prob, setup = helpers.oracle_problem_from_gpu(fg, wl, dev)
        o_tr, o_hist = orc.forward(prob, np.float32)
        rng = np.random.default_rng(nx + ny + pml)
        resid = rng.standard_normal(o_tr.shape).astype(np.float32)
        oe, os_ = orc.adjoint_reference(prob, o_hist, resid, np.float64)
        er, se, mr = (torch.tensor(np.ascontiguousarray(a), device=dev) for a in (wl.er, wl.se, wl.mr))
        for tuning in TUNINGS:
            solve = fg.Solve(dev, setup, tv=False, tuning=tuning)
            traces, hist = solve.forward(er, se, mr)
            ge, gs = solve.gradient(er, se, mr, hist, torch.tensor(resid, device=dev), normalize=False)
            solve.plan.device_check()
            tag = "%dx%d pml %d tuning %s" % (nx, ny, pml, tuning)
            assert np.array_equal(traces.cpu().numpy(), o_tr), "traces differ: " + tag
            assert helpers.rel_l2(ge.cpu().numpy(), oe) < 1e-6, "g_eps: " + tag
            assert helpers.rel_l2(gs.cpu().numpy(), os_) < 1e-6, "g_sig: " + tag
            n += 1
    print("ok %d" % n)


if __name__ == "__main__":
    main()
