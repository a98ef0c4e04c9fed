"""CPU oracle: ctypes wrapper of fdtd_oracle.cpp plus an FP64 restatement of
the reference's host-side set-up.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, never by the shipped package.  It is the
checker the CUDA path is compared against.

Parity pin: the oracle is checked against the reference's own CUDA kernels
(built from the reference sources into oracle/_ref/ and driven by
oracle/ref_driver.py on a GPU host) and against golden vectors generated from
them (tests/golden/).  The reference itself ships no tests or golden data.

FP64 set-up restated from the reference (paths relative to that project):
  update coefficients   src/lib/uc.cu:21-38 (ucget), :70-87 (ucgeta)
  CPML profile          src/compute.py:80-123 (sigma_max, quartic grading)
  HORIPML coefficients  src/compute.py:212-222
  Ricker waveform       src/compute.py:383-400, scaled as sourcereceiver.cu:75
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

EPS0 = 8.8541878128e-12
MU0 = 1.25663706212e-06
Z0 = (MU0 / EPS0) ** 0.5


class _OracleProblem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("th", ctypes.c_int), ("S", ctypes.c_int),
        ("nt", ctypes.c_int), ("nrx", ctypes.c_int), ("nsrc", ctypes.c_int), ("dtype", ctypes.c_int),
        ("d", ctypes.c_double), ("dt", ctypes.c_double),
        ("uE0", ctypes.c_void_p), ("uE1", ctypes.c_void_p), ("uE4", ctypes.c_void_p),
        ("uH1", ctypes.c_void_p), ("uH4", ctypes.c_void_p), ("uE0a", ctypes.c_void_p),
        ("pml", ctypes.c_void_p), ("src", ctypes.c_void_p), ("srcw", ctypes.c_void_p), ("rx", ctypes.c_void_p),
    ]


_libs = {}


def build() -> None:
    """Compile the oracle with its Makefile (g++, no GPU needed)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib(variant: str = "") -> ctypes.CDLL:
    name = "liboracle%s.so" % variant
    if name not in _libs:
        path = os.path.join(BUILD, name)
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_forward.argtypes = [ctypes.POINTER(_OracleProblem), ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_forward.restype = ctypes.c_int
        L.oracle_adjoint_ref.argtypes = [ctypes.POINTER(_OracleProblem), ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_adjoint_ref.restype = ctypes.c_int
        L.oracle_adjoint_exact.argtypes = [ctypes.POINTER(_OracleProblem), ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_adjoint_exact.restype = ctypes.c_int
        L.oracle_step.argtypes = [ctypes.POINTER(_OracleProblem), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.oracle_step.restype = ctypes.c_int
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_set_threads.restype = ctypes.c_int
        _libs[name] = L
    return _libs[name]


def set_threads(n: int) -> int:
    return _lib().oracle_set_threads(int(n))


def positions2(pos3: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """(S, n, 3) cell indices -> (S, n, 2) with -1 marking inert cells
    (the zero frame i == nx / j == ny and the dead k == 1 plane)."""
    pos3 = np.asarray(pos3, dtype=np.int64)
    out = pos3[..., :2].astype(np.int32).copy()
    inert = (pos3[..., 2] != 0) | (pos3[..., 0] >= nx) | (pos3[..., 1] >= ny)
    out[inert] = -1
    return np.ascontiguousarray(out)


@dataclass
class Problem:
    """One model, S shots.  Coefficient arrays are (nx, ny); pml is (8, th)."""
    nx: int
    ny: int
    th: int
    shots: int
    nt: int
    d: float
    dt: float
    uE0: np.ndarray
    uE1: np.ndarray
    uE4: np.ndarray
    uH1: np.ndarray
    uH4: np.ndarray
    uE0a: np.ndarray
    pml: Optional[np.ndarray]
    src: np.ndarray     # (S, nsrc, 2) int32
    srcw: np.ndarray    # (nsrc, nt)
    rx: np.ndarray      # (S, nrx, 2) int32

    def cast(self, dtype) -> "Problem":
        c = lambda a: np.ascontiguousarray(a, dtype=dtype)
        return Problem(self.nx, self.ny, self.th, self.shots, self.nt, self.d, self.dt,
                       c(self.uE0), c(self.uE1), c(self.uE4), c(self.uH1), c(self.uH4), c(self.uE0a),
                       None if self.pml is None else c(self.pml),
                       np.ascontiguousarray(self.src, dtype=np.int32), c(self.srcw),
                       np.ascontiguousarray(self.rx, dtype=np.int32))


def _struct(p: Problem, dtype):
    keep = [p]
    s = _OracleProblem()
    s.nx, s.ny, s.th, s.S, s.nt = p.nx, p.ny, p.th, p.shots, p.nt
    s.nrx, s.nsrc = p.rx.shape[1], p.src.shape[1]
    s.dtype = 0 if dtype == np.float32 else 1
    s.d, s.dt = float(p.d), float(p.dt)
    s.uE0, s.uE1, s.uE4 = p.uE0.ctypes.data, p.uE1.ctypes.data, p.uE4.ctypes.data
    s.uH1, s.uH4, s.uE0a = p.uH1.ctypes.data, p.uH4.ctypes.data, p.uE0a.ctypes.data
    s.pml = p.pml.ctypes.data if p.pml is not None and p.pml.size else None
    s.src, s.srcw, s.rx = p.src.ctypes.data, p.srcw.ctypes.data, p.rx.ctypes.data
    return s, keep


def forward(p: Problem, dtype=np.float32, keep_history=True, variant: str = ""):
    """Returns (traces (S, nt, nrx), hist (nt, S, nx, ny) or None)."""
    q = p.cast(dtype)
    s, keep = _struct(q, dtype)
    traces = np.zeros((q.shots, q.nt, q.rx.shape[1]), dtype=dtype)
    hist = np.zeros((q.nt, q.shots, q.nx, q.ny), dtype=dtype) if keep_history else None
    rc = _lib(variant).oracle_forward(ctypes.byref(s), traces.ctypes.data,
                                      hist.ctypes.data if hist is not None else None)
    if rc:
        raise RuntimeError("oracle_forward failed: %d" % rc)
    return traces, hist


def adjoint_reference(p: Problem, hist: np.ndarray, resid: np.ndarray, dtype=np.float32, variant: str = ""):
    """Unnormalised reference-mode imaging sums (g_eps, g_sig), each (nx, ny)."""
    q = p.cast(dtype)
    s, keep = _struct(q, dtype)
    h = np.ascontiguousarray(hist, dtype=dtype)
    g = np.ascontiguousarray(resid, dtype=dtype)
    ge = np.zeros((q.nx, q.ny), dtype=dtype)
    gs = np.zeros((q.nx, q.ny), dtype=dtype)
    rc = _lib(variant).oracle_adjoint_ref(ctypes.byref(s), h.ctypes.data, g.ctypes.data, ge.ctypes.data,
                                          gs.ctypes.data)
    if rc:
        raise RuntimeError("oracle_adjoint_ref failed: %d" % rc)
    return ge, gs


def exact_sums(p: Problem, hist: np.ndarray, w: np.ndarray, dtype=np.float64):
    """Imaging sums of the exact discrete adjoint for J = sum w * traces:
    s1 = sum_t lambda_t Ez(x_{t-1}), s2 = sum_t lambda_t Ez(x_t), each (nx, ny)."""
    q = p.cast(dtype)
    s, keep = _struct(q, dtype)
    h = np.ascontiguousarray(hist, dtype=dtype)
    g = np.ascontiguousarray(w, dtype=dtype)
    s1 = np.zeros((q.nx, q.ny), dtype=dtype)
    s2 = np.zeros((q.nx, q.ny), dtype=dtype)
    rc = _lib().oracle_adjoint_exact(ctypes.byref(s), h.ctypes.data, g.ctypes.data, s1.ctypes.data, s2.ctypes.data)
    if rc:
        raise RuntimeError("oracle_adjoint_exact failed: %d" % rc)
    return s1, s2


def exact_gradient(s1, s2, er, se, dt):
    """Gradient of J with respect to (eps_r, sigma) from the exact sums.

    Step t-1 makes Ez_t = c0 Ez_{t-1} + uE4 q on a cell whose E is updated by
    the leapfrog (i, j >= 1; c0 = uE0 = EB/EA) and Ez_t = Ez_{t-1} + uE4 q on
    the CPML-only cells of rows / columns 0 (c0 = 1), with EA = a er + se/2,
    EB = a er - se/2, a = e0/dt (e0 the float32 constant of uc.cu:8) and uE4 =
    1/EA.  Differentiating the coefficients with q fixed:
      d/der: (a/EA) (Ez_{t-1} - Ez_t)
      d/dse: -(Ez_{t-1} + Ez_t) / (2 EA)  (leapfrog cells), -(Ez_t - Ez_{t-1}) / (2 EA) (row/column 0)
    times lambda_t, summed over t and shots.  PEC cells (se > 100) get 0."""
    er = np.asarray(er, dtype=np.float64)
    se = np.asarray(se, dtype=np.float64)
    a = float(np.float32(EPS0)) / dt
    EA = a * er + 0.5 * se
    ge = (a / EA) * (s1 - s2)
    gs = -(s1 + s2) / (2 * EA)
    edge = np.zeros(er.shape, dtype=bool)
    edge[0, :] = True
    edge[:, 0] = True
    gs[edge] = (-(s2 - s1) / (2 * EA))[edge]
    pec = se > 100
    ge[pec] = 0.0
    gs[pec] = 0.0
    return ge, gs


def state_size(p: Problem) -> int:
    """Length of a packed state vector (oracle_step's packing)."""
    F = (p.nx + 1) * (p.ny + 1)
    return p.shots * (3 * F + 4 * p.th * p.ny + 4 * p.nx * p.th)


def frame_mask(p: Problem) -> np.ndarray:
    """1 on the packed state's entries that are part of the solution space
    (fields on i < nx, j < ny; every CPML auxiliary), 0 on the zero frame."""
    F = (p.nx + 1) * (p.ny + 1)
    f = np.zeros((p.nx + 1, p.ny + 1))
    f[:p.nx, :p.ny] = 1.0
    field = np.tile(f.reshape(-1), p.shots)
    rest = np.ones(state_size(p) - 3 * p.shots * F)
    return np.concatenate([field, field, field, rest])


def step(p: Problem, state: np.ndarray, transpose: bool = False, dtype=np.float64) -> np.ndarray:
    """One source-free time step of a packed state (or its transpose)."""
    q = p.cast(dtype)
    s, keep = _struct(q, dtype)
    x = np.ascontiguousarray(state, dtype=dtype)
    out = np.zeros_like(x)
    rc = _lib().oracle_step(ctypes.byref(s), x.ctypes.data, out.ctypes.data, 1 if transpose else 0)
    if rc:
        raise RuntimeError("oracle_step failed: %d" % rc)
    return out


# ---------------------------------------------------------------------------
# FP64 set-up (the same equations in double precision)
# ---------------------------------------------------------------------------

def coefficients_fp64(er, se, mr, dt, dx):
    """ucget / ucgeta in double precision.  Returns dict of (nx, ny) arrays."""
    er = np.asarray(er, dtype=np.float64)
    se = np.asarray(se, dtype=np.float64)
    mr = np.asarray(mr, dtype=np.float64)
    e0 = float(np.float32(EPS0))
    m0 = float(np.float32(MU0))
    HA = m0 * mr / dt
    uH1 = (1.0 / dx) / HA
    uH4 = 1.0 / HA
    EA = e0 * er / dt + 0.5 * se
    EB = e0 * er / dt - 0.5 * se
    pec = se > 100
    uE0 = np.where(pec, 0.0, EB / EA)
    uE1 = np.where(pec, 0.0, (1.0 / dx) / EA)
    uE4 = np.where(pec, 0.0, 1.0 / EA)
    uE0a = np.where(pec, 0.0, (2 * e0 * er) / (2 * e0 * er + se * dt))
    return dict(uE0=uE0, uE1=uE1, uE4=uE4, uH1=uH1, uH4=uH4, uE0a=uE0a)


def cpml_fp64(th: int, d: float, er_avg: float, mr_avg: float, dt: float) -> np.ndarray:
    """(8, th) HORIPML coefficients in double precision."""
    if th <= 0:
        return np.zeros((8, 0))
    order = 4
    smax = (0.8 * (order + 1)) / (Z0 * d * math.sqrt(er_avg * mr_avg))
    k = np.arange(th, dtype=np.float64)
    esig = (k / th) ** order * smax
    hsig = ((k + 0.5) / th) ** order * smax
    two_e0 = 2 * EPS0

    def hor(sig):
        tmp = two_e0 + dt * sig
        return [two_e0 / tmp, two_e0 / tmp, (two_e0 - dt * sig) / tmp, (2 * sig * dt) / tmp]

    return np.array(hor(esig) + hor(hsig))


def ricker_fp64(nt: int, dt: float, time_window: float, amp: float, freq: float, d: float) -> np.ndarray:
    """Ricker on whole steps times dl/(dx dy dz) = 1/d^2, double precision."""
    chi = math.sqrt(2.0) / freq
    zeta = math.pi ** 2 * freq ** 2
    t = dt * np.arange(nt)
    delay = t - chi
    w = -(2 * zeta * (2 * zeta * delay ** 2 - 1) * np.exp(-zeta * delay ** 2)) / (2 * zeta) * amp
    w[(t < 0) | (t > time_window)] = 0.0
    return w * d / (d * d * d)
