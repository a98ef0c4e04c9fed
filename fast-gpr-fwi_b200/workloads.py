"""Seeded synthetic GPR workloads for the benchmark configurations.

No public dataset is involved.  Each generator builds a physical model
(depth along reference axis 0, distance along axis 1), pads it by the CPML
thickness on every side with edge replication (as the reference notebook
does, example.ipynb cell 0), and returns the keyword arguments of
``compute()``.  Positions are in compute-grid metres (physical metres plus
the pad), dt = 0.95 x CFL and time_windows = (nt - 1.5) dt so that the
solve has exactly nt steps.

  config 0  140x100 (100x60 + 2x20), dx 0.1 m,    1 shot,  nt 1200, 20 rx, 100 MHz
  config 1  240x160 (200x120 + 2x20), dx 0.05 m,  13 shots, nt 3000, 40 rx, 100 MHz
  config 2  440x340 (400x300 + 2x20), dx 0.025 m, 64 shots, nt 4000, 100 rx, 200 MHz
  config 3  840x540 (800x500 + 2x20), dx 0.02 m,  30 shots, nt 6000, 120 rx, 50/100/200 MHz
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

C0 = 299792458.0
PAD = 20


@dataclass
class Workload:
    name: str
    nx: int            # compute grid, axis 0 (with CPML pad)
    ny: int            # compute grid, axis 1
    dx: float
    shots: int
    nt: int
    freq: float
    er: np.ndarray     # (nx, ny) float32
    se: np.ndarray
    mr: np.ndarray
    source_location: list
    source_step: list
    receiver_location: list
    receiver_step: list
    nrx: int
    fixed_receiver: bool = True
    pml: int = PAD
    er_init: Optional[np.ndarray] = None
    se_init: Optional[np.ndarray] = None
    extra: dict = field(default_factory=dict)

    @property
    def dt(self) -> float:
        return 0.95 * self.dx / (C0 * math.sqrt(2.0))

    @property
    def cell_steps(self) -> int:
        return self.nx * self.ny * self.shots * self.nt

    def kwargs(self, device, er=None, se=None, mr=None, tv=True, **over):
        """Arguments of compute() for this workload (tensors on `device`)."""
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a)[:, :, None], device=device)
        kw = dict(
            device=device, dx=self.dx, ny=self.ny, nx=self.nx, nz=1,
            source=["hertzian", "z"], source_apmlitudes=["ricker", 1, self.freq], step=self.shots,
            er=t(self.er) if er is None else er, se=t(self.se) if se is None else se,
            mr=t(self.mr) if mr is None else mr,
            nsrc=1, nrx=self.nrx, time_windows=(self.nt - 1.5) * self.dt,
            source_location=torch.tensor(self.source_location, dtype=torch.float32),
            source_step=torch.tensor(self.source_step, dtype=torch.float32),
            receiver_location=torch.tensor(self.receiver_location, dtype=torch.float32),
            receiver_step=torch.tensor(self.receiver_step, dtype=torch.float32),
            pmlthick=self.pml, dt=self.dt, tv=tv, Fixedreceiver=self.fixed_receiver,
        )
        kw.update(over)
        return kw


def _pad(a: np.ndarray, p: int) -> np.ndarray:
    return np.pad(a, p, mode="edge")


def _gaussian_model(rng, nz: int, nx: int, dx: float):
    """eps_r = 4 + 3 Gaussian anomalies, sigma = 2e-3 + co-located anomalies."""
    z = (np.arange(nz) + 0.5) * dx
    x = (np.arange(nx) + 0.5) * dx
    Z, X = np.meshgrid(z, x, indexing="ij")
    er = np.full((nz, nx), 4.0)
    se = np.full((nz, nx), 2e-3)
    for _ in range(3):
        a = rng.uniform(-1.0, 8.0)
        w = rng.uniform(0.3, 1.0)
        cz, cx = rng.uniform(0, nz * dx), rng.uniform(0, nx * dx)
        g = np.exp(-((Z - cz) ** 2 + (X - cx) ** 2) / (2 * w * w))
        er += a * g
        se += rng.uniform(1e-3, 1e-2) * g
    return np.maximum(er, 1.0), se


def config0(seed: int = 1000) -> Workload:
    rng = np.random.default_rng(seed)
    dx = 0.1
    er, se = _gaussian_model(rng, 100, 60, dx)
    p = PAD * dx
    return Workload("config0", 140, 100, dx, 1, 1200, 1e8,
                    _pad(er, PAD).astype(np.float32), _pad(se, PAD).astype(np.float32),
                    np.ones((140, 100), np.float32),
                    source_location=[5.0 + p, 1.0 + p, 0.0], source_step=[0.0, 0.0, 0.0],
                    receiver_location=[0.25 + p, 5.0 + p, 0.0], receiver_step=[0.5, 0.0, 0.0], nrx=20)


def config1(seed: int = 1001) -> Workload:
    rng = np.random.default_rng(seed)
    dx = 0.05
    er, se = _gaussian_model(rng, 200, 120, dx)
    from scipy.ndimage import gaussian_filter
    er_i = gaussian_filter(er, 10.0, mode="nearest")
    se_i = gaussian_filter(se, 10.0, mode="nearest")
    p = PAD * dx
    f = lambda a: _pad(a, PAD).astype(np.float32)
    return Workload("config1", 240, 160, dx, 13, 3000, 1e8, f(er), f(se), np.ones((240, 160), np.float32),
                    source_location=[0.5 + p, 0.5 + p, 0.0], source_step=[0.75, 0.0, 0.0],
                    receiver_location=[0.125 + p, 5.5 + p, 0.0], receiver_step=[0.25, 0.0, 0.0], nrx=40,
                    er_init=f(er_i), se_init=f(se_i))


def _layered_model(rng, nz: int, nx: int, dx: float):
    """5-8 dipping interfaces (eps_r ~ U[3,15] per layer, sigma log-uniform in
    [1e-4, 2e-2] per layer) plus 2-4 Gaussian lenses."""
    z = (np.arange(nz) + 0.5) * dx
    x = (np.arange(nx) + 0.5) * dx
    Z, X = np.meshgrid(z, x, indexing="ij")
    n_if = int(rng.integers(5, 9))
    depth = nz * dx
    base = np.sort(rng.uniform(0.1 * depth, 0.9 * depth, n_if))
    dips = rng.uniform(-0.15, 0.15, n_if)
    layer = np.zeros((nz, nx), dtype=np.int64)
    for k in range(n_if):
        layer += (Z > base[k] + dips[k] * (X - 0.5 * nx * dx)).astype(np.int64)
    eps_l = rng.uniform(3.0, 15.0, n_if + 1)
    sig_l = np.exp(rng.uniform(np.log(1e-4), np.log(2e-2), n_if + 1))
    er = eps_l[layer]
    se = sig_l[layer]
    for _ in range(int(rng.integers(2, 5))):
        a = rng.uniform(-2.0, 4.0)
        w = rng.uniform(0.2, 0.6)
        cz, cx = rng.uniform(0, depth), rng.uniform(0, nx * dx)
        g = np.exp(-((Z - cz) ** 2 + (X - cx) ** 2) / (2 * w * w))
        er = er + a * g
    return np.clip(er, 1.0, 20.0), se


def config2(seed: int = 1002, shots: int = 64, nt: int = 4000) -> Workload:
    rng = np.random.default_rng(seed)
    dx = 0.025
    er, se = _layered_model(rng, 400, 300, dx)
    p = PAD * dx
    f = lambda a: _pad(a, PAD).astype(np.float32)
    return Workload("config2", 440, 340, dx, shots, nt, 2e8, f(er), f(se), np.ones((440, 340), np.float32),
                    source_location=[0.1 + p, 0.5 + p, 0.0], source_step=[0.15, 0.0, 0.0],
                    receiver_location=[0.05 + p, 7.0 + p, 0.0], receiver_step=[0.1, 0.0, 0.0], nrx=100)


def config3(seed: int = 1003, freq: float = 2e8) -> Workload:
    rng = np.random.default_rng(seed)
    dx = 0.02
    er, se = _layered_model(rng, 800, 500, dx)
    p = PAD * dx
    f = lambda a: _pad(a, PAD).astype(np.float32)
    return Workload("config3", 840, 540, dx, 30, 6000, freq, f(er), f(se), np.ones((840, 540), np.float32),
                    source_location=[0.5 + p, 0.5 + p, 0.0], source_step=[0.5, 0.0, 0.0],
                    receiver_location=[0.4 + p, 9.5 + p, 0.0], receiver_step=[0.125, 0.0, 0.0], nrx=120)


def small(seed: int = 7, nx: int = 48, ny: int = 40, shots: int = 3, nt: int = 120, pml: int = 6,
          dx: float = 0.05, nrx: int = 9, fixed: bool = False) -> Workload:
    """A small seeded case for parity tests (seconds on the CPU oracle)."""
    rng = np.random.default_rng(seed)
    er, se = _gaussian_model(rng, nx - 2 * pml, ny - 2 * pml, dx)
    er = _pad(er, pml).astype(np.float32)
    se = _pad(se, pml).astype(np.float32)
    p = pml * dx
    return Workload("small", nx, ny, dx, shots, nt, 6e8, er, se, np.ones((nx, ny), np.float32),
                    source_location=[p + 0.3, p + 0.25, 0.0], source_step=[0.25, 0.05, 0.0],
                    receiver_location=[p + 0.1, ny * dx - p - 0.3, 0.0], receiver_step=[0.15, 0.0, 0.0],
                    nrx=nrx, fixed_receiver=fixed, pml=pml)


CONFIGS = {"config0": config0, "config1": config1, "config2": config2, "config3": config3}
