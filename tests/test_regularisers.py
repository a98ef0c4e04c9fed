"""TV regulariser and multiscale FIR against golden vectors produced by the
reference's own src/tv.py and src/multiscale.py (tests/golden/make_golden_cpu.py)."""
import os

import numpy as np
import pytest
import torch

from conftest import HERE

GOLD = np.load(os.path.join(HERE, "golden", "ref_tv_fir.npz"))


@pytest.mark.parametrize("key", ["tv_in32", "tv_in64", "tv_sig_in"])
def test_tv_matches_reference(fg, key):
    out_key = {"tv_in32": "tv_out32", "tv_in64": "tv_out64", "tv_sig_in": "tv_sig_out"}[key]
    x = torch.tensor(GOLD[key])
    got = fg.total_variation(x.clone()).numpy()
    want = GOLD[out_key]
    assert got.shape == want.shape
    # the four-neighbour sum is a conv2d in the reference: its summation order
    # differs from ours by rounding only
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5 * np.abs(want).max())


@pytest.mark.parametrize("fs,fc", [(1e10, 1e8), (1e10, 2.5e8), (8e9, 1e8), (1.25e10, 2e8)])
def test_fir_design_matches_reference(fg, fs, fc):
    key = "fir_%d_%d_taps" % (int(fs / 1e6), int(fc / 1e6))
    got = fg.design_fir_filter(fc, fs, int(fs / fc)).numpy()
    np.testing.assert_array_equal(got, GOLD[key])


def test_fir_apply_matches_reference(fg):
    got3 = fg.apply_filter(torch.tensor(GOLD["fir_data3"]), 1e10, 1e8).numpy()
    np.testing.assert_allclose(got3, GOLD["fir_out3"], rtol=1e-6, atol=1e-6)
    got1 = fg.apply_filter(torch.tensor(GOLD["fir_data1"]), 8e9, 1e8).numpy()
    np.testing.assert_allclose(got1, GOLD["fir_out1"], rtol=1e-6, atol=1e-6)
    with pytest.raises(ValueError):
        fg.apply_filter(torch.zeros(2, 3), 1e10, 1e8)
