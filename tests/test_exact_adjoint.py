"""The exact discrete adjoint on the CPU oracle (FP64): the transpose of one
time step passes the dot-product test, and the gradient it gives agrees with
centred finite differences of the forward loop."""
import numpy as np
import pytest

import helpers


def _cases(fg):
    tiny = fg.workloads.small(seed=11, shots=3, nt=90, nx=17, ny=33, pml=8, nrx=4)
    tiny.source_location = [0.45, 0.45, 0.0]
    tiny.source_step = [0.05, 0.1, 0.0]
    tiny.receiver_location = [0.3, 1.2, 0.0]
    tiny.receiver_step = [0.1, 0.0, 0.0]
    return [fg.workloads.small(), fg.workloads.small(seed=3, shots=2, nt=150, nx=40, ny=56, pml=5, nrx=6), tiny]


@pytest.mark.parametrize("case", range(3))
def test_step_transpose_dot_product(fg, orc, case):
    wl = _cases(fg)[case]
    prob, _ = helpers.oracle_problem_cpu(wl)
    p64 = prob.cast(np.float64)
    rng = np.random.default_rng(case)
    m = orc.frame_mask(p64)
    x = rng.standard_normal(orc.state_size(p64)) * m
    y = rng.standard_normal(orc.state_size(p64)) * m
    a = np.dot(orc.step(p64, x) * m, y)
    b = np.dot(x, orc.step(p64, y, transpose=True) * m)
    assert abs(a - b) <= 1e-12 * abs(a), (a, b)


@pytest.mark.parametrize("case", range(3))
def test_exact_gradient_vs_centred_fd(fg, orc, case):
    """<grad J, delta> against (J(m + h delta) - J(m - h delta)) / 2h in FP64,
    for J = sum w * traces, with h scaled to each parameter (eps_r ~ 4, sigma ~
    1e-3 S/m) and perturbations everywhere, CPML included."""
    wl = _cases(fg)[case]
    prob, setup = helpers.oracle_problem_cpu(wl)
    er = np.maximum(wl.er, 1).astype(np.float64)
    se = np.maximum(wl.se, 0).astype(np.float64)
    rng = np.random.default_rng(100 + case)
    w = rng.standard_normal((wl.shots, setup.nt, wl.nrx))

    def J(e, s):
        tr, _ = orc.forward(helpers.fp64_problem(prob, setup, wl, e, s), np.float64, keep_history=False)
        return float(np.sum(w * tr))

    p64 = helpers.fp64_problem(prob, setup, wl, er, se)
    _, hist = orc.forward(p64, np.float64)
    s1, s2 = orc.exact_sums(p64, hist, w)
    ge, gs = orc.exact_gradient(s1, s2, er, se, setup.dt32)
    smooth = helpers.bump(wl.nx, wl.ny, wl.nx / 2, wl.ny / 2, 5.0)
    for de, ds, h in ((smooth, 0 * smooth, 1e-3), (0 * smooth, smooth, 1e-6),
                      (rng.standard_normal(er.shape), 0 * smooth, 1e-4),
                      (0 * smooth, rng.standard_normal(er.shape), 1e-7)):
        fd = (J(er + h * de, se + h * ds) - J(er - h * de, se - h * ds)) / (2 * h)
        ad = float(np.sum(ge * de) + np.sum(gs * ds))
        assert abs(fd - ad) <= 1e-5 * abs(fd), (fd, ad)


def test_exact_adjoint_fp32_stays_finite_config0(fg, orc):
    """Config 0 (CPML 20 cells, 1200 steps): the FP32 exact adjoint stays
    finite and within 1e-4 of the FP64 one.  Row 0 and column 0 are closed
    CPML-only subsystems that the forward never excites; unprojected, their
    transposed recursion overflows FP32 after a few hundred steps."""
    wl = fg.workloads.config0()
    prob, setup = helpers.oracle_problem_cpu(wl)
    rng = np.random.default_rng(34)
    w = rng.standard_normal((wl.shots, wl.nt, wl.nrx))
    _, h32 = orc.forward(prob, np.float32)
    a1, a2 = orc.exact_sums(prob, h32, w.astype(np.float32), dtype=np.float32)
    assert np.isfinite(a1).all() and np.isfinite(a2).all()
    _, h64 = orc.forward(prob, np.float64)
    b1, b2 = orc.exact_sums(prob, h64, w)
    er, se = np.maximum(wl.er, 1), np.maximum(wl.se, 0)
    g32 = orc.exact_gradient(a1.astype(np.float64), a2.astype(np.float64), er, se, setup.dt32)
    g64 = orc.exact_gradient(b1, b2, er, se, setup.dt32)
    for x, y in zip(g32, g64):
        assert helpers.rel_l2(x, y) < 1e-4
