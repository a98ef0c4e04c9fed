"""Host-side set-up (grid.py) against the FP64 restatement and the
reference's rules for dt, iteration count and position rounding."""
import math

import numpy as np
import pytest
import torch

import helpers


def test_iterations_and_dt(fg):
    g = helpers.grid_mod()
    wl = fg.workloads.config0()
    setup = helpers.setup_for(wl, torch.device("cpu"))
    assert setup.nt == wl.nt
    assert setup.dt == wl.dt
    assert g.iteration_count(torch.tensor(1e-7), 1e-10, "cpu") == 1001   # the reference notebook's case
    cfl = g.cfl_dt(0.05)
    assert g.choose_dt(0.05, None) == cfl
    assert g.choose_dt(0.05, 2 * cfl) == cfl
    assert g.choose_dt(0.05, 0.5 * cfl) == 0.5 * cfl
    assert abs(cfl - 0.05 / (299792458.0 * math.sqrt(2))) < 1e-22


def test_positions_round_half_even(fg):
    g = helpers.grid_mod()
    idx = g.grid_positions(4, torch.tensor([2.25, 7.0, 0.0]), torch.tensor([0.5, 0.0, 0.0]), 1, 0.1, "cpu")
    # 22.5 -> 22, 27.5 -> 28 (torch.round is half-to-even)
    assert idx[0, :, 0].tolist() == [22, 28, 32, 38]
    assert idx[0, :, 1].tolist() == [70, 70, 70, 70]
    moving = g.grid_positions(2, torch.tensor([1.0, 1.0, 0.0]), torch.tensor([0.5, 0.0, 0.0]), 3, 0.1, "cpu")
    assert moving[:, 0, 0].tolist() == [10, 15, 20]
    fixed = g.grid_positions(2, torch.tensor([1.0, 1.0, 0.0]), torch.tensor([0.5, 0.0, 0.0]), 3, 0.1, "cpu",
                             fixed=True)
    assert fixed[:, 0, 0].tolist() == [10, 10, 10]


def test_waveform_matches_fp64(fg, orc):
    wl = fg.workloads.config0()
    setup = helpers.setup_for(wl, torch.device("cpu"))
    tw = (wl.nt - 1.5) * wl.dt
    ref = orc.ricker_fp64(setup.nt, setup.dt, tw, 1.0, wl.freq, setup.dx)
    got = setup.srcw[0].astype(np.float64)
    assert np.abs(got - ref).max() < 2e-6 * np.abs(ref).max()
    assert setup.srcw[0, -1] == 0.0   # last step lies beyond the time window


def test_cpml_profile_matches_fp64(fg, orc):
    wl = fg.workloads.config0()
    setup = helpers.setup_for(wl, torch.device("cpu"))
    er_avg = float(np.mean(wl.er[0, :].astype(np.float64)))
    ref = orc.cpml_fp64(setup.th, setup.dx, er_avg, 1.0, setup.dt32)
    got = setup.profile.packed().astype(np.float64)
    np.testing.assert_allclose(got, ref, rtol=5e-6, atol=1e-6)
    # first E cell of each slab has zero conductivity: RA=RB=RE=1, RF=0
    assert got[0, 0] == 1 and got[2, 0] == 1 and got[3, 0] == 0


def test_coefficients_f32_vs_fp64(fg, orc):
    wl = fg.workloads.small()
    f32 = helpers.coefficients_f32(wl.er, wl.se, wl.mr, 1e-10, 0.05)
    f64 = orc.coefficients_fp64(wl.er, wl.se, wl.mr, float(np.float32(1e-10)), float(np.float32(0.05)))
    for k in f32:
        np.testing.assert_allclose(f32[k], f64[k], rtol=2e-6)


def test_bad_inputs_raise(fg):
    wl = fg.workloads.small()
    kw = wl.kwargs("cpu")
    with pytest.raises(ValueError):
        fg.compute(**dict(kw, nz=2))
    with pytest.raises(ValueError):
        fg.compute(**dict(kw, pml_formulation="MRIPML"))
    with pytest.raises(ValueError):
        fg.compute(**dict(kw, source_apmlitudes=["gaussian", 1, 1e8]))
    with pytest.raises(RuntimeError):
        fg.compute(**kw)   # no CUDA device: the solver never falls back to the CPU
