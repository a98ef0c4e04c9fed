"""The TV regulariser kernel (fg_total_variation) against the tensor
restatement of the reference's src/tv.py and the reference's golden vectors."""
import os
from importlib import import_module

import numpy as np
import pytest
import torch

from conftest import HERE

GOLD = np.load(os.path.join(HERE, "golden", "ref_tv_fir.npz"))
gpu = pytest.mark.gpu


def _models():
    rng = np.random.default_rng(11)
    smooth = np.cumsum(np.cumsum(rng.standard_normal((120, 90)), 0), 1).astype(np.float32)
    layered = np.repeat(rng.uniform(3, 15, size=(12, 1)), 20, axis=0) * np.ones((1, 70))
    layered = (layered + 0.3 * rng.standard_normal(layered.shape)).astype(np.float32)
    thin = rng.uniform(1, 9, size=(1, 17)).astype(np.float32)
    return {"smooth": smooth, "layered": layered, "thin_row": thin, "thin_col": thin.T.copy(),
            "gold32": GOLD["tv_in32"][:, :, 0], "gold_sig": GOLD["tv_sig_in"][:, :, 0]}


def _mods():
    return import_module("fast-gpr-fwi_b200.tv"), import_module("fast-gpr-fwi_b200._native")


@gpu
@pytest.mark.parametrize("name", list(_models()))
@pytest.mark.parametrize("num_iter", [0, 1, 7, 60])
def test_tv_kernel_bit_exact_fixed_iterations(fg, name, num_iter):
    """With tol = 0 both run exactly num_iter iterations: identical bits."""
    tvm, nat = _mods()
    x = _models()[name]
    want = tvm._total_variation_tensor(torch.tensor(x), 0.02, 1.0, num_iter, 0.0)[:, :, 0].numpy()
    got, iters = nat.total_variation(torch.tensor(x, device="cuda"), 0.02, 1.0, num_iter, 0.0)
    assert iters == num_iter
    np.testing.assert_array_equal(got.cpu().numpy(), want)


@gpu
@pytest.mark.parametrize("lamda,rho", [(0.02, 1.0), (0.05, 2.0), (1e-3, 0.5)])
def test_tv_kernel_scalars(fg, lamda, rho):
    tvm, nat = _mods()
    x = _models()["smooth"]
    want = tvm._total_variation_tensor(torch.tensor(x), lamda, rho, 25, 0.0)[:, :, 0].numpy()
    got, _ = nat.total_variation(torch.tensor(x, device="cuda"), lamda, rho, 25, 0.0)
    np.testing.assert_array_equal(got.cpu().numpy(), want)


@gpu
@pytest.mark.parametrize("key", ["tv_in32", "tv_sig_in"])
def test_tv_drop_in_on_cuda_matches_reference(fg, key):
    """The drop-in entry point on a CUDA tensor (default arguments, early
    stop) against the reference's own output."""
    out_key = {"tv_in32": "tv_out32", "tv_sig_in": "tv_sig_out"}[key]
    x = torch.tensor(GOLD[key], device="cuda")
    got = fg.total_variation(x)
    assert got.is_cuda and tuple(got.shape) == GOLD[out_key].shape
    assert tuple(x.shape) == GOLD[key].shape[:2]          # the reference squeezes its argument in place
    want = GOLD[out_key]
    # the reference sums the four neighbours with a conv2d: rounding differs
    np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-5, atol=1e-5 * np.abs(want).max())


@gpu
def test_tv_drop_in_default_stop_matches_tensor_path(fg):
    """Default tol on a model of the size the gradient regularises
    (440 x 340): the same result as the tensor path."""
    rng = np.random.default_rng(3)
    x = (6 + np.cumsum(rng.standard_normal((440, 340)), 1) * 0.05).astype(np.float32)
    cpu = fg.total_variation(torch.tensor(x)[:, :, None]).numpy()
    got = fg.total_variation(torch.tensor(x, device="cuda")[:, :, None]).cpu().numpy()
    np.testing.assert_allclose(got, cpu, rtol=1e-6, atol=1e-6 * np.abs(cpu).max())


# --- multiscale FIR (fg_fir_causal) ---------------------------------------

@gpu
def test_fir_kernel_matches_reference_golden(fg):
    got3 = fg.apply_filter(torch.tensor(GOLD["fir_data3"], device="cuda"), 1e10, 1e8)
    assert got3.is_cuda and tuple(got3.shape) == GOLD["fir_out3"].shape
    np.testing.assert_allclose(got3.cpu().numpy(), GOLD["fir_out3"], rtol=1e-6, atol=1e-6)
    got1 = fg.apply_filter(torch.tensor(GOLD["fir_data1"], device="cuda"), 8e9, 1e8)
    np.testing.assert_allclose(got1.cpu().numpy(), GOLD["fir_out1"], rtol=1e-6, atol=1e-6)


@gpu
@pytest.mark.parametrize("shape,fs,fc", [((64, 4000, 100), 1.78e10, 2e8), ((3, 257, 7), 1e10, 2.5e8),
                                         ((2, 50, 1), 1e10, 2e8), ((1, 31, 33), 1e10, 3.3e8)])
def test_fir_kernel_matches_tensor_path(fg, shape, fs, fc):
    rng = np.random.default_rng(2)
    x = rng.standard_normal(shape).astype(np.float32)
    want = fg.apply_filter(torch.tensor(x), fs, fc).numpy()          # CPU: the reference's tensor arithmetic
    got = fg.apply_filter(torch.tensor(x, device="cuda"), fs, fc).cpu().numpy()
    scale = np.abs(want).max()
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6 * scale)


@gpu
def test_fir_kernel_rejects_padding_longer_than_series(fg):
    nat = __import__("importlib").import_module("fast-gpr-fwi_b200._native")
    with pytest.raises(nat.FastGprError):
        nat.fir_causal(torch.zeros((1, 10, 2), device="cuda"), torch.ones(11))
