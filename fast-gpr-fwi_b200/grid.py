"""Host-side set-up of one FDTD solve: time step, positions, waveform, CPML.

Everything here is O(nx + ny + nt) scalar work done once per ``compute()``
call; the per-cell work (update coefficients, time stepping, imaging) happens
in the CUDA library.  The arithmetic follows the reference's set-up code step
for step, with the same dtypes and the same op order, so that the integer
positions and iteration count are identical and the float32 coefficient
profiles are identical bit for bit:

  time step / CFL / iterations   src/compute.py:752-803
  source / receiver positions    src/compute.py:774-796
  Ricker waveform                src/compute.py:334-357, 383-400
  CPML sigma_max and profile     src/compute.py:80-123, 267-313
  HORIPML update coefficients    src/compute.py:193-222 (forward branch; the
                                 adjoint branch is unreachable because
                                 PML.adjoint is hard-set False at :152)
  Hertzian-dipole scaling        src/lib/sourcereceiver.cu:73-75
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

# scipy.constants values (CODATA 2018), the constants the reference imports.
C0 = 299792458.0
EPS0 = 8.8541878128e-12
MU0 = 1.25663706212e-06
Z0 = (MU0 / EPS0) ** 0.5  # src/__init__.py:21

def cfl_dt(dx):
    """Courant limit of the 2-D TMz leapfrog, compute.py:754.

    Evaluated with the caller's dx object (Python float or 0-d tensor), in the
    reference's operation order, so the result has the reference's type too.
    """
    inv = 1 / dx
    return 1 / (C0 * (((inv * inv) + (inv * inv)) ** 0.5))


def choose_dt(dx, dt):
    """dt selection of compute.py:752-769: CFL when dt is None or too large."""
    limit = cfl_dt(dx)
    if dt is None:
        return limit
    if dt > limit:
        print(limit)
        print(dt)
        print("dt is too large")
        return limit
    return dt


def iteration_count(time_windows, dt, device) -> int:
    """compute.py:798-803: int(ceil(tw/dt)) + 1 with tw as a float32 tensor."""
    if not isinstance(time_windows, torch.Tensor):
        time_windows = torch.tensor(time_windows, device=device)
    return int(torch.ceil(time_windows / dt)) + 1


def grid_positions(count, location, step_vec, shots, dx, device, fixed=False):
    """Cell indices of a line of `count` points per shot, compute.py:774-796.

    Point n of shot s sits at location + n*step + s*step (metres) and is
    rounded with torch.round(pos/dx) on the solve's device.  Returns an int32
    tensor (shots, count, 3) on `device`.
    """
    pos = torch.zeros((shots, count, 3), device=device)
    for c in range(3):
        pos[:, :, c] = (torch.arange(count, device=device) * step_vec[c] + location[c]).repeat(shots, 1)
    shift = torch.arange(pos.size(0), device=device).view(-1, 1, 1) * (step_vec.to(device))
    pos = pos + shift
    idx = torch.round(pos / dx).int().contiguous()
    if fixed:
        idx[:, :, :] = idx[0, :, :].unsqueeze(0)
    return idx


def ricker_scaled(nt: int, dt, time_window, amp, freq, d32: np.float32) -> np.ndarray:
    """Ricker samples on whole steps times the Hertzian-dipole factor.

    Waveform: compute.py:351-357 with Waveform.calculate_value (:391-400),
    float32 CPU tensor arithmetic in the reference's op order (torch's CPU
    exp, whose vectorised and 0-d forms agree element for element).
    Scaling: sourcereceiver.cu:73-75, w * dl / (dx * dy * dz) with dl = dz
    and dx = dy = dz in float32.
    """
    f32 = torch.float32
    freq_t = torch.tensor(float(freq), dtype=f32)
    amp_t = torch.tensor(float(amp), dtype=f32)
    chi = torch.sqrt(torch.tensor(2.0)) / freq_t
    zeta = (math.pi ** 2) * (freq_t ** 2)
    z2 = 2 * zeta
    normalise = 1 / z2
    tw = torch.tensor(float(time_window), dtype=f32)
    if isinstance(dt, torch.Tensor):
        t = (dt.to(f32) * torch.arange(nt, dtype=f32))
    else:
        t = torch.tensor(float(dt) * np.arange(nt, dtype=np.float64), dtype=f32)
    delay = t - chi
    d2 = delay ** 2
    v = -(z2 * (z2 * d2 - 1) * torch.exp(-zeta * d2)) * normalise
    v = v * amp_t
    v = torch.where((t >= 0) & (t <= tw), v, torch.zeros_like(v))
    d = torch.tensor(float(d32), dtype=f32)
    return ((v * d) / ((d * d) * d)).numpy()


def slab_average(values: torch.Tensor) -> torch.Tensor:
    """Mean of one slab face as build_pmls computes it (compute.py:278-283).

    A sequential running sum in the tensor's dtype, then multiplied by the
    float reciprocal of the count (CUDA's division by a host scalar).  Returns
    a 0-d CPU tensor of the input dtype.
    """
    v = values.detach().reshape(-1).cpu().numpy()
    dt = v.dtype.type
    acc = dt(0)
    for x in v:
        acc = dt(acc + x)
    inv = dt(1) / dt(v.size)
    return torch.tensor(acc * inv)


@dataclass
class CPMLProfile:
    """HORIPML coefficients of one slab (all four slabs are identical)."""
    thickness: int
    sigma_max: float
    ERA: np.ndarray
    ERB: np.ndarray
    ERE: np.ndarray
    ERF: np.ndarray
    HRA: np.ndarray
    HRB: np.ndarray
    HRE: np.ndarray
    HRF: np.ndarray

    def packed(self) -> np.ndarray:
        """(8, th) float32: ERA ERB ERE ERF HRA HRB HRE HRF."""
        return np.stack([self.ERA, self.ERB, self.ERE, self.ERF,
                         self.HRA, self.HRB, self.HRE, self.HRF]).astype(np.float32)


def cpml_profile(th: int, d, er_avg: torch.Tensor, mr_avg: torch.Tensor, dt) -> CPMLProfile:
    """sigma_max (compute.py:80-84), quartic grading (:86-123), HORIPML (:212-222).

    The reference computes sigma_max once, from the first slab built (x0), and
    the CFS object is shared by all slabs (compute.py:178-179, :829), so the
    four slabs carry the same coefficient vectors.
    """
    order = 4
    smax = (0.8 * (order + 1)) / (Z0 * d * torch.sqrt(er_avg * mr_avg))
    n = th + 1
    grading = (torch.linspace(0, (n - 1) + 0.5, steps=2 * n) / (n - 1)) ** order
    e_prof = grading[0:-1:2]
    h_prof = grading[1::2]
    smax32 = torch.tensor(float(smax), dtype=torch.float32)
    esig = (e_prof * smax32)[:-1]
    hsig = (h_prof * smax32)[:-1]
    dt32 = torch.tensor(float(dt), dtype=torch.float32)
    two_e0 = torch.tensor(2 * EPS0, dtype=torch.float32)

    def horipml(sig):
        loss = dt32 * sig
        tmp = two_e0 + loss
        ra = two_e0 / tmp
        rb = two_e0 / tmp
        re = (two_e0 - loss) / tmp
        rf = ((2 * sig) * dt32) / tmp
        return ra.numpy(), rb.numpy(), re.numpy(), rf.numpy()

    ERA, ERB, ERE, ERF = horipml(esig)
    HRA, HRB, HRE, HRF = horipml(hsig)
    return CPMLProfile(th, float(smax), ERA, ERB, ERE, ERF, HRA, HRB, HRE, HRF)


@dataclass
class SolveSetup:
    """Everything the CUDA library needs besides the material arrays."""
    nx: int
    ny: int
    shots: int
    nt: int
    dx: float                    # float32 value of the cell size
    dt: object                   # dt as the reference returns it (float or tensor)
    dt32: float                  # float32 value handed to the kernels
    th: int
    src: torch.Tensor            # (shots, nsrc, 3) int32, device
    rx: torch.Tensor             # (shots, nrx, 3) int32, device
    srcw: np.ndarray             # (nsrc, nt) float32 scaled source waveforms
    profile: Optional[CPMLProfile] = None
    freq: object = None
    extra: dict = field(default_factory=dict)


def _as_int(v) -> int:
    return int(v.item()) if isinstance(v, torch.Tensor) else int(v)


def build_setup(device, dx, ny, nx, nz, time_windows, source, source_location, source_step,
                receiver_location, receiver_step, pmlthick, source_amplitudes, step, er, mr,
                nsrc, nrx, dt, freq, total_step, fixed_receiver, customsource, customreceiver) -> SolveSetup:
    """The geometry part of the reference's initialization(), compute.py:726-830."""
    nx_i, ny_i, nz_i = _as_int(nx), _as_int(ny), _as_int(nz)
    if nz_i != 1:
        raise ValueError("only the 2-D TMz mode (nz == 1) is supported; got nz=%d" % nz_i)
    if nx_i < 2 or ny_i < 2:
        raise ValueError("grid must be at least 2x2 cells")
    shots = _as_int(step)
    if shots < 1:
        raise ValueError("step (shots) must be >= 1")
    ts = shots if total_step is None else _as_int(total_step)
    g_dt = choose_dt(dx, dt)
    nt = iteration_count(time_windows, g_dt, device)
    if nt < 1:
        raise ValueError("time window gives no time steps")
    tw = time_windows if isinstance(time_windows, torch.Tensor) else torch.tensor(time_windows)

    if customsource is None:
        src = grid_positions(nsrc, source_location, source_step, ts, dx, device)
    else:
        src = customsource
    if customreceiver is None:
        rx = grid_positions(nrx, receiver_location, receiver_step, ts, dx, device, fixed=fixed_receiver)
    else:
        rx = customreceiver
    src = src[:shots].to(torch.int32).contiguous()
    rx = rx[:shots].to(torch.int32).contiguous()

    if source[1] != "z":
        raise ValueError("only z-polarised Hertzian dipoles exist in TMz mode")
    wtype = source_amplitudes[0]
    if wtype != "ricker":
        raise ValueError("waveform type %r is not supported (reference supports 'ricker')" % (wtype,))
    d32 = np.float32(float(dx))
    w = ricker_scaled(nt, g_dt, tw, source_amplitudes[1], source_amplitudes[2], d32)
    srcw = np.zeros((max(int(nsrc), 1), nt), dtype=np.float32)
    srcw[0] = w   # only waveform row 0 is ever filled (compute.py:561-564)

    th = _as_int(pmlthick)
    if th < 0 or 2 * th > min(nx_i, ny_i):
        raise ValueError("pmlthick must be in [0, min(nx, ny)/2]")
    profile = None
    if th > 0:
        er_avg = slab_average(er[0, :ny_i, :nz_i])
        mr_avg = slab_average(mr[0, :ny_i, :nz_i])
        profile = cpml_profile(th, dx, er_avg, mr_avg, g_dt)

    return SolveSetup(nx=nx_i, ny=ny_i, shots=shots, nt=nt, dx=float(d32), dt=g_dt,
                      dt32=float(np.float32(float(g_dt))), th=th, src=src, rx=rx,
                      srcw=srcw, profile=profile, freq=freq)
