"""Shared helpers of the test suite: problem construction for the oracle."""
from __future__ import annotations

import importlib

import numpy as np
import torch

from oracle import oracle as orc

PKG = "fast-gpr-fwi_b200"


def grid_mod():
    return importlib.import_module(PKG + ".grid")


def native_mod():
    return importlib.import_module(PKG + "._native")


def setup_for(wl, device, er=None, mr=None):
    """The package's host set-up (grid.build_setup) for a workload."""
    kw = wl.kwargs(device)
    er = kw["er"] if er is None else er
    mr = kw["mr"] if mr is None else mr
    er = torch.clamp(er, min=1)
    return grid_mod().build_setup(
        kw["device"], kw["dx"], kw["ny"], kw["nx"], kw["nz"], kw["time_windows"], kw["source"],
        kw["source_location"], kw["source_step"], kw["receiver_location"], kw["receiver_step"],
        kw["pmlthick"], kw["source_apmlitudes"], kw["step"], er, mr, kw["nsrc"], kw["nrx"], kw["dt"],
        None, None, kw["Fixedreceiver"], None, None)


def coefficients_f32(er, se, mr, dt, dx):
    """numpy float32 restatement of the reference's ucget/ucgeta
    (src/lib/uc.cu:21-38, :70-87) -- the CPU-side stand-in for the
    coefficient kernel.  The adjoint denominator is one fused multiply-add,
    emulated through float64 (exact product)."""
    f = np.float32
    er, se, mr = (np.asarray(a, dtype=f) for a in (er, se, mr))
    dt, dx = f(dt), f(dx)
    e0, m0 = f(8.8541878128e-12), f(1.25663706212e-06)
    HA = (m0 * mr) / dt
    inv_dx = f(1) / dx
    uH1 = inv_dx / HA
    uH4 = f(1) / HA
    q = (e0 * er) / dt
    hs = 0.5 * se.astype(np.float64)
    EA = (q.astype(np.float64) + hs).astype(f)
    EB = (q.astype(np.float64) - hs).astype(f)
    pec = se > 100
    z = f(0)
    uE0 = np.where(pec, z, EB / EA)
    uE1 = np.where(pec, z, inv_dx / EA)
    uE4 = np.where(pec, z, f(1) / EA)
    num = (f(2) * e0) * er
    den = (se.astype(np.float64) * float(dt) + num.astype(np.float64)).astype(f)
    uE0a = np.where(pec, z, num / den)
    return dict(uE0=uE0, uE1=uE1, uE4=uE4, uH1=uH1, uH4=uH4, uE0a=uE0a)


def make_problem(setup, coef, nx, ny):
    pml = setup.profile.packed() if setup.profile is not None else np.zeros((8, 0), np.float32)
    return orc.Problem(nx, ny, setup.th, setup.shots, setup.nt, setup.dx, setup.dt32,
                       coef["uE0"], coef["uE1"], coef["uE4"], coef["uH1"], coef["uH4"], coef["uE0a"], pml,
                       orc.positions2(setup.src.cpu().numpy(), nx, ny), setup.srcw,
                       orc.positions2(setup.rx.cpu().numpy(), nx, ny))


def oracle_problem_cpu(wl):
    """Oracle problem with CPU-emulated float32 coefficients."""
    setup = setup_for(wl, torch.device("cpu"))
    coef = coefficients_f32(np.maximum(wl.er, 1), np.maximum(wl.se, 0), wl.mr, setup.dt32, setup.dx)
    return make_problem(setup, coef, wl.nx, wl.ny), setup


def oracle_problem_from_gpu(fg, wl, dev):
    """Oracle problem whose coefficients come from the package's CUDA kernel."""
    setup = setup_for(wl, dev)
    nat = native_mod()
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)
    er, se, mr = t(np.maximum(wl.er, 1)), t(np.maximum(wl.se, 0)), t(wl.mr)
    cf = nat.coefficients(er, se, mr, setup.dt32, setup.dx, adjoint=False).cpu().numpy()
    ca = nat.coefficients(er, se, mr, setup.dt32, setup.dx, adjoint=True).cpu().numpy()
    nx, ny = wl.nx, wl.ny
    coef = dict(uE0=cf[0, :nx, :ny], uE1=cf[1, :nx, :ny], uE4=cf[2, :nx, :ny], uH1=cf[3, :nx, :ny],
                uH4=cf[4, :nx, :ny], uE0a=ca[0, :nx, :ny])
    return make_problem(setup, coef, nx, ny), setup


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def fp64_problem(prob, setup, wl, er=None, se=None):
    """The oracle problem in double precision with the set-up restated in FP64
    (coefficients, CPML profile, Ricker) -- the FP64 oracle of the same update
    equations.  er / se override the workload's model (the CPML profile keeps
    the workload's, so that it stays fixed under a model perturbation)."""
    er = np.maximum(wl.er, 1) if er is None else er
    se = np.maximum(wl.se, 0) if se is None else se
    f64 = orc.coefficients_fp64(er, se, wl.mr, setup.dt32, setup.dx)
    p64 = prob.cast(np.float64)
    for k, v in f64.items():
        setattr(p64, k, v)
    er_avg = float(np.mean(np.maximum(wl.er, 1)[0, :].astype(np.float64)))
    p64.pml = orc.cpml_fp64(setup.th, setup.dx, er_avg, 1.0, setup.dt32)
    p64.srcw = np.zeros_like(prob.srcw, dtype=np.float64)
    p64.srcw[0] = orc.ricker_fp64(setup.nt, setup.dt32, (wl.nt - 1.5) * wl.dt, 1.0, wl.freq, setup.dx)
    return p64


def bump(nx, ny, ci, cj, width):
    """Smooth (nx, ny) perturbation: a Gaussian of the given width (cells)."""
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    return np.exp(-(((i - ci) / width) ** 2 + ((j - cj) / width) ** 2))


def run_package(fg, wl, dev, w, tuning=None, tv=False, adjoint="reference"):
    """compute() + backward of sum(w * traces): (traces, g_eps, g_sig) on the device."""
    er = torch.tensor(np.ascontiguousarray(wl.er[:, :, None]), device=dev, requires_grad=True)
    se = torch.tensor(np.ascontiguousarray(wl.se[:, :, None]), device=dev, requires_grad=True)
    traces, dt = fg.compute(**wl.kwargs(dev, er=er, se=se, tv=tv, tuning=tuning, adjoint=adjoint))
    (traces * w).sum().backward()
    torch.cuda.synchronize()
    return traces.detach(), er.grad[:, :, 0].detach(), se.grad[:, :, 0].detach()


def run_reference(refdrv, wl, dev, w):
    """The reference's CUDA kernels driven as its Python driver drives them
    (oracle/ref_driver.py): (grid, traces, g_eps, g_sig)."""
    kw = wl.kwargs(dev)
    er = torch.clamp(kw["er"], min=1)
    se = torch.clamp(kw["se"], min=0)
    G = refdrv.setup(dev, kw["dx"], kw["ny"], kw["nx"], 1, kw["time_windows"], kw["source_location"],
                     kw["source_step"], kw["receiver_location"], kw["receiver_step"], kw["pmlthick"],
                     kw["source_apmlitudes"], kw["step"], er, se, kw["mr"], kw["nsrc"], kw["nrx"], kw["dt"],
                     kw["Fixedreceiver"])
    rxs, hist = refdrv.forward(G)
    ge, gs = refdrv.backward(G, er, se, kw["mr"], hist, w)
    return G, rxs[:, 2].contiguous(), ge[:, :, 0], gs[:, :, 0]


def edge_workload(fg, nx, ny, pml, shots=3, nt=60):
    """A small seeded case on an nx x ny grid with `pml` CPML cells, the
    source and receivers inside the grid."""
    wl = fg.workloads.small(seed=nx * 100 + ny + pml, nx=nx, ny=ny, shots=shots, nt=nt, pml=min(pml, 6) if pml else 0,
                            nrx=3)
    wl.pml = pml
    dx = wl.dx
    wl.source_location = [dx * (nx // 3), dx * (ny // 3), 0.0]
    wl.source_step = [dx, 0.0, 0.0] if shots < nx // 3 else [0.0, 0.0, 0.0]
    wl.receiver_location = [dx * (nx // 2), dx * (2 * ny // 3), 0.0]
    wl.receiver_step = [dx, 0.0, 0.0]
    return wl
