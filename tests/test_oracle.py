"""The CPU oracle on its own: FP32 vs FP64 agreement and the properties of
the reference algorithm it restates."""
import numpy as np
import pytest

import helpers


@pytest.fixture(scope="module")
def small_case(fg):
    wl = fg.workloads.small()
    prob, setup = helpers.oracle_problem_cpu(wl)
    return wl, prob, setup


def test_fp32_tracks_fp64(orc, small_case):
    wl, prob, setup = small_case
    tr32, h32 = orc.forward(prob, np.float32)
    tr64, h64 = orc.forward(prob, np.float64)
    assert np.abs(tr64).max() > 0
    assert helpers.rel_l2(tr32, tr64) < 1e-5
    resid = tr64 * 0.5
    ge32, gs32 = orc.adjoint_reference(prob, h32, resid, np.float32)
    ge64, gs64 = orc.adjoint_reference(prob, h64, resid, np.float64)
    assert helpers.rel_l2(ge32, ge64) < 1e-5 and helpers.rel_l2(gs32, gs64) < 1e-5


def test_first_sample_zero_and_history_consistent(orc, small_case):
    """trace[t] is Ez after step t-1 (store_outputs runs first, compute.py:578)."""
    wl, prob, setup = small_case
    tr, hist = orc.forward(prob, np.float64)
    assert np.all(tr[:, 0, :] == 0)
    for s in range(prob.shots):
        for r in range(prob.rx.shape[1]):
            i, j = prob.rx[s, r]
            if i >= 0:
                np.testing.assert_array_equal(tr[s, 1:, r], hist[:-1, s, i, j])


def test_linearity_in_source(orc, small_case):
    """Doubling the waveform doubles the traces (exact in binary FP up to the
    final rounding)."""
    wl, prob, setup = small_case
    tr1, _ = orc.forward(prob, np.float64, keep_history=False)
    p2 = prob.cast(np.float64)
    p2.srcw = p2.srcw * 2.0
    tr2, _ = orc.forward(p2, np.float64, keep_history=False)
    np.testing.assert_allclose(tr2, 2 * tr1, rtol=1e-12, atol=1e-12 * np.abs(tr1).max())


def test_shots_independent(orc, small_case):
    """A shot computed alone equals the same shot inside a batch."""
    wl, prob, setup = small_case
    trb, _ = orc.forward(prob, np.float32, keep_history=False)
    for s in range(prob.shots):
        p1 = prob.cast(np.float32)
        p1.shots = 1
        p1.src = np.ascontiguousarray(prob.src[s:s + 1])
        p1.rx = np.ascontiguousarray(prob.rx[s:s + 1])
        tr1, _ = orc.forward(p1, np.float32, keep_history=False)
        np.testing.assert_array_equal(tr1[0], trb[s])


def test_cpml_absorbs(orc, fg):
    """With the CPML, energy leaving the grid does not come back: late-time
    traces are far smaller than with the CPML switched off (th=0 reflects)."""
    wl = fg.workloads.small(nt=800, pml=8, nx=64, ny=64)
    prob, setup = helpers.oracle_problem_cpu(wl)
    tr, _ = orc.forward(prob, np.float64, keep_history=False)
    p0 = prob.cast(np.float64)
    p0.th = 0
    p0.pml = np.zeros((8, 0))
    tr0, _ = orc.forward(p0, np.float64, keep_history=False)
    late = slice(600, 800)
    assert np.abs(tr[:, late]).max() < 0.2 * np.abs(tr0[:, late]).max()
