"""The launch-shape autotuner: it returns a valid shape for the geometry,
caches it, and the tuned solve computes the default solve's bits."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shots", [40, 3])
def test_autotune_picks_a_valid_shape_with_identical_results(fg, shots):
    at = importlib.import_module("fast-gpr-fwi_b200.autotune")
    dev = torch.device("cuda:0")
    wl = fg.workloads.small(shots=shots, nt=90, nx=64, ny=56, fixed=True)
    wl.source_step = [0.03, 0.01, 0.0]
    res = []
    for tuning in (None, "auto"):
        er = torch.tensor(wl.er[:, :, None], device=dev, requires_grad=True)
        se = torch.tensor(wl.se[:, :, None], device=dev, requires_grad=True)
        tr, _ = fg.compute(**wl.kwargs(dev, er=er, se=se, tv=False, tuning=tuning))
        (tr ** 2).sum().backward()
        torch.cuda.synchronize()
        res.append((tr.detach().cpu().numpy(), er.grad.cpu().numpy(), se.grad.cpu().numpy()))
    for a, b in zip(*res):
        assert np.array_equal(a, b)
    assert len(at._CACHE) >= 1
    tuned = next(iter(at._CACHE.values()))
    nat = __import__("importlib").import_module("fast-gpr-fwi_b200._native")
    assert set(tuned) <= set(nat.FgTuning.KEYS)
