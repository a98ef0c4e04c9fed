"""The CPU oracle against golden vectors produced by the reference's own CUDA
kernels (tests/golden/make_golden.py, run on a GPU host with the kernels
compiled from the reference sources).  This pins the oracle: fed with the
reference's coefficient planes, CPML vectors and positions, its float32
forward reproduces the reference traces bit for bit, and its reference-mode
adjoint reproduces the reference's (unnormalised) imaging sums."""
import os

import numpy as np
import pytest

import helpers
from conftest import HERE

CASES = ["small", "small_moving", "config0"]


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", "ref_%s.npz" % name)))


def problem(orc, g):
    nx, ny = int(g["nx"]), int(g["ny"])
    return orc.Problem(nx, ny, int(g["th"]), int(g["shots"]), int(g["nt"]), float(g["dx"]), float(g["dt"]),
                       g["uE0"], g["uE1"], g["uE4"], g["uH1"], g["uH4"], g["uE0a"], g["pml"],
                       orc.positions2(g["src"], nx, ny), _scaled_waveform(g), orc.positions2(g["rx"], nx, ny))


def _scaled_waveform(g):
    d = np.float32(g["dx"])
    w = np.zeros((g["src"].shape[1], int(g["nt"])), np.float32)
    w[0] = (g["waveform"] * d) / ((d * d) * d)
    return w


@pytest.mark.parametrize("name", CASES)
def test_oracle_forward_bit_exact_vs_reference(orc, name):
    g = load(name)
    tr, _ = orc.forward(problem(orc, g), np.float32, keep_history=False)
    np.testing.assert_array_equal(tr, g["traces"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_adjoint_vs_reference(orc, name):
    g = load(name)
    p = problem(orc, g)
    _, hist = orc.forward(p, np.float32)
    ge, gs = orc.adjoint_reference(p, hist, g["resid"], np.float64)
    assert helpers.rel_l2(ge, g["ge"]) < 1e-5
    assert helpers.rel_l2(gs, g["gs"]) < 1e-5


@pytest.mark.parametrize("name", CASES)
def test_host_setup_vs_reference(fg, name):
    """The package's float32 set-up reproduces the reference's waveform and
    CPML vectors (positions are compared on the GPU, where the reference
    computes them)."""
    g = load(name)
    wl = {"small": fg.workloads.small(), "config0": fg.workloads.config0(),
          "small_moving": fg.workloads.small(seed=3, shots=2, nt=150, nx=40, ny=56, pml=5, nrx=6)}[name]
    setup = helpers.setup_for(wl, "cpu")
    assert setup.nt == int(g["nt"])
    np.testing.assert_array_equal(setup.srcw[0], _scaled_waveform(g)[0])
    np.testing.assert_array_equal(setup.profile.packed(), g["pml"])
    coef = helpers.coefficients_f32(g["er"], g["se"], g["mr"], float(g["dt"]), float(g["dx"]))
    for k in ("uE0", "uE1", "uE4", "uH1", "uH4"):
        np.testing.assert_array_equal(coef[k], g[k])
    ulp = np.abs(coef["uE0a"].view(np.int32).astype(np.int64) - g["uE0a"].view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
