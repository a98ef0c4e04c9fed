"""Drive the reference's own CUDA kernels (oracle/_ref/*.so) the way the
reference's Python driver does.

TEST INFRASTRUCTURE ONLY (GPU hosts).  The shared objects are compiled from
the reference sources by ``make -C oracle ref`` with the reference's own
nvcc flags; this module restates, in the same order and with the same torch
dtype/device semantics, the host code around them (paths relative to the
reference project):

  initialization()      src/compute.py:726-872
  build_pmls / CFS      src/compute.py:54-313
  Forward()             src/compute.py:542-720
  backinitialization()  src/compute.py:945-1017
  Backward()            src/compute.py:1020-1180

It is the parity target for the package: traces, imaging gradients and
coefficient planes produced here are what "the reference" means in the GPU
parity tests and in tests/golden/.
"""
from __future__ import annotations

import ctypes
import decimal
import math
import os
from collections import OrderedDict

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

C0 = 299792458.0
EPS0 = 8.8541878128e-12
MU0 = 1.25663706212e-06
Z0 = (MU0 / EPS0) ** 0.5

_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int)
_libs = None


def available() -> bool:
    names = ["fields_updates_gpu", "sourcereceiver", "uc", "pml_updates_h", "pml_updates_e", "back"]
    return all(os.path.exists(os.path.join(REF_DIR, n + ".so")) for n in names)


def libs():
    """Load the six reference libraries and declare their signatures
    (the argtypes of src/__init__.py:39-221)."""
    global _libs
    if _libs is not None:
        return _libs
    L = {n: ctypes.cdll.LoadLibrary(os.path.join(REF_DIR, n + ".so"))
         for n in ["fields_updates_gpu", "sourcereceiver", "uc", "pml_updates_h", "pml_updates_e", "back"]}
    i, f = ctypes.c_int, ctypes.c_float
    pml_args = [i] * 13 + [_F] * 12 + [f, _F] + [i] * 4
    for lib in (L["pml_updates_e"], L["pml_updates_h"]):
        for d in ("xminus", "xplus", "yminus", "yplus"):
            fn = getattr(lib, "order1_" + d)
            fn.argtypes = pml_args
            fn.restype = None
    fu = L["fields_updates_gpu"]
    for name in ("e_fields_updates", "h_fields_updates"):
        getattr(fu, name).argtypes = [_F] * 8 + [i] * 4
        getattr(fu, name).restype = None
    sr = L["sourcereceiver"]
    sr.launch_store_outputs.argtypes = [i, i, i, _I] + [_F] * 7 + [i] * 6
    sr.launch_store_outputs.restype = None
    src_args = [i, i, f, f, f, _I, f, _F, _F, _F, _F, _F, i, i, i, i, i, i]
    sr.update_hertzian_dipole.argtypes = src_args
    sr.update_hertzian_dipole.restype = None
    L["back"].back_source.argtypes = src_args
    L["back"].back_source.restype = None
    for name in ("Ucget", "Ucgeta"):
        getattr(L["uc"], name).argtypes = [_F] * 9 + [i, i, i, f, f]
        getattr(L["uc"], name).restype = None
    _libs = L
    return L


def fp(t: torch.Tensor):
    return ctypes.cast(t.data_ptr(), _F)


def ip(t: torch.Tensor):
    return ctypes.cast(t.data_ptr(), _I)


# ---------------------------------------------------------------------------
# set-up (compute.py:54-313, 726-872)
# ---------------------------------------------------------------------------

class _CFS:
    def __init__(self, device):
        self.sigma_max = None
        self.device = device

    def values(self, th, which):
        if which == "sigma":
            n = th + 1
            tmp = (torch.linspace(0, (n - 1) + 0.5, steps=2 * n) / (n - 1)) ** 4
            E = tmp[0:-1:2].to(self.device)
            H = tmp[1::2].to(self.device)
            E = E * (self.sigma_max - 0) + 0
            H = H * (self.sigma_max - 0) + 0
        else:
            c = 0.0 if which == "alpha" else 1.0
            E = torch.zeros(th + 1, device=self.device) + c
            H = torch.zeros(th + 1, device=self.device) + c
        return E[:-1], H[:-1]


class _Slab:
    def __init__(self, direction, xs, xf, ys, yf, zs, zf, d):
        self.direction = direction
        self.xs, self.xf, self.ys, self.yf, self.zs, self.zf = xs, xf, ys, yf, zs, zf
        self.nx, self.ny, self.nz = xf - xs, yf - ys, zf - zs
        self.d = d
        self.thickness = self.nx if direction[0] == "x" else self.ny


def _build_pmls(G, er, mr):
    cfs = _CFS(G.device)
    G.pmls = []
    for key, value in G.pmlthickness.items():
        if value <= 0:
            continue
        sumer = 0
        summr = 0
        if key[0] == "x":
            if key == "x0":
                pml = _Slab("xminus", 0, value, 0, G.ny, 0, G.nz, G.dx)
            else:
                pml = _Slab("xplus", G.nx - value, G.nx, 0, G.ny, 0, G.nz, G.dx)
            for j in range(int(G.ny)):
                for k in range(int(G.nz)):
                    sumer += er[pml.xs, j, k]
                    summr += mr[pml.xs, j, k]
            averageer = sumer / (G.ny * G.nz)
            averagemr = summr / (G.ny * G.nz)
        elif key[0] == "y":
            if key == "y0":
                pml = _Slab("yminus", 0, G.nx, 0, value, 0, G.nz, G.dy)
            else:
                pml = _Slab("yplus", 0, G.nx, G.ny - value, G.ny, 0, G.nz, G.dy)
            for i in range(int(G.nx)):
                for k in range(int(G.nz)):
                    sumer += er[i, pml.ys, k]
                    summr += mr[i, pml.ys, k]
            averageer = sumer / (G.nx * G.nz)
            averagemr = summr / (G.nx * G.nz)
        else:
            continue
        G.pmls.append(pml)
        if not cfs.sigma_max:
            cfs.sigma_max = (0.8 * (4 + 1)) / (Z0 * pml.d * torch.sqrt(averageer * averagemr))
        Ealpha, Halpha = cfs.values(pml.thickness, "alpha")
        Ekappa, Hkappa = cfs.values(pml.thickness, "kappa")
        Esigma, Hsigma = cfs.values(pml.thickness, "sigma")
        dt = G.dt
        tmp = (2 * EPS0 * Ekappa) + dt * (Ealpha * Ekappa + Esigma)
        pml.ERA = ((2 * EPS0 + dt * Ealpha) / tmp).view(1, -1).contiguous()
        pml.ERB = ((2 * EPS0 * Ekappa) / tmp).view(1, -1).contiguous()
        pml.ERE = (((2 * EPS0 * Ekappa) - dt * (Ealpha * Ekappa + Esigma)) / tmp).view(1, -1).contiguous()
        pml.ERF = ((2 * Esigma * dt) / (Ekappa * tmp)).view(1, -1).contiguous()
        tmp = (2 * EPS0 * Hkappa) + dt * (Halpha * Hkappa + Hsigma)
        pml.HRA = ((2 * EPS0 + dt * Halpha) / tmp).view(1, -1).contiguous()
        pml.HRB = ((2 * EPS0 * Hkappa) / tmp).view(1, -1).contiguous()
        pml.HRE = (((2 * EPS0 * Hkappa) - dt * (Halpha * Hkappa + Hsigma)) / tmp).view(1, -1).contiguous()
        pml.HRF = ((2 * Hsigma * dt) / (Hkappa * tmp)).view(1, -1).contiguous()


def _alloc_phi(G):
    for p in G.pmls:
        S, dev = G.step, G.device
        nx, ny, nz = p.nx, p.ny, p.nz
        if p.direction[0] == "x":
            shapes = [(S, nx + 1, ny, nz + 1), (S, nx + 1, ny + 1, nz), (S, nx, ny + 1, nz), (S, nx, ny, nz + 1)]
        else:
            shapes = [(S, nx, ny + 1, nz + 1), (S, nx + 1, ny + 1, nz), (S, nx + 1, ny, nz), (S, nx, ny, nz + 1)]
        p.EPhi1, p.EPhi2, p.HPhi1, p.HPhi2 = [torch.zeros(s, device=dev) for s in shapes]


def _coefficients(G, er, se, mr, adjoint):
    L = libs()
    dev = G.device
    shape = (int(G.nx) + 1, int(G.ny) + 1, int(G.nz) + 1)
    c = [torch.zeros(shape, device=dev) for _ in range(6)]
    ere = torch.zeros(shape, device=dev)
    ere[:G.nx, :G.ny, :G.nz] = er
    see = torch.zeros(shape, device=dev)
    see[:G.nx, :G.ny, :G.nz] = se
    mre = torch.zeros(shape, device=dev)
    mre[:G.nx, :G.ny, :G.nz] = mr
    fn = L["uc"].Ucgeta if adjoint else L["uc"].Ucget
    fn(fp(ere), fp(see), fp(mre), *[fp(x) for x in c], shape[0], shape[1], shape[2], G.dt, G.dx)
    G.uE0, G.uE1, G.uE4, G.uH0, G.uH1, G.uH4 = [x.unsqueeze(0).repeat(G.step, 1, 1, 1) for x in c]
    G.coef_single = c


class Grid:
    pass


def setup(device, dx, ny, nx, nz, time_windows, source_location, source_step, receiver_location,
          receiver_step, pmlthick, source_amplitudes, step, er, se, mr, nsrc, nrx, dt=None,
          Fixedreceiver=False):
    """initialization() of compute.py:726-872 (HORIPML, Ricker, no custom tables)."""
    se = torch.clamp(se, min=0, max=1e6)
    G = Grid()
    G.step, G.device, G.dx, G.dy, G.dz = step, device, dx, dx, dx
    G.nx, G.ny, G.nz, G.nrx, G.nsrc = nx, ny, nz, nrx, nsrc
    cfl = 1 / (C0 * ((((1 / G.dx) * (1 / G.dx)) + ((1 / G.dy) * (1 / G.dy))) ** 0.5))
    G.dt = cfl if (dt is None or dt > cfl) else dt
    G.pmlthickness = OrderedDict((k, 10) for k in ["x0", "y0", "z0", "xmax", "ymax", "zmax"])
    G.pmlthickness["z0"] = 0
    G.pmlthickness["zmax"] = 0
    ts = step
    src = torch.zeros((ts, nsrc, 3), device=device)
    for c in range(3):
        src[:, :, c] = (torch.arange(nsrc, device=device) * source_step[c] + source_location[c]).repeat(ts, 1)
    src = src + torch.arange(src.size(0), device=device).view(-1, 1, 1) * source_step.to(device)
    G.source = torch.round(src / G.dx).int().contiguous()
    rx = torch.zeros((ts, nrx, 3), device=device)
    for c in range(3):
        rx[:, :, c] = (torch.arange(nrx, device=device) * receiver_step[c] + receiver_location[c]).repeat(ts, 1)
    rx = rx + torch.arange(rx.size(0), device=device).view(-1, 1, 1) * receiver_step.to(device)
    G.receiver = torch.round(rx / G.dx).int().contiguous()
    if Fixedreceiver:
        G.receiver[:, :, :] = G.receiver[0, :, :].unsqueeze(0)
    if not isinstance(time_windows, torch.Tensor):
        time_windows = torch.tensor(time_windows, device=device)
    G.iterations = int(torch.ceil(time_windows / G.dt)) + 1
    for k in ("x0", "y0", "xmax", "ymax"):
        G.pmlthickness[k] = pmlthick
    # Ricker on whole steps, compute.py:351-357, 383-400
    amp = torch.tensor(source_amplitudes[1], dtype=torch.float)
    freq = torch.tensor(source_amplitudes[2], dtype=torch.float)
    tw = time_windows.clone().detach()
    w = torch.zeros((G.iterations), device=device)
    chi = torch.sqrt(torch.tensor(2.0)) / freq
    zeta = (torch.pi ** 2) * (freq ** 2)
    for it in range(G.iterations):
        t = G.dt * it
        if t >= 0 and t <= tw:
            delay = t - chi
            normalise = 1 / (2 * zeta)
            v = -(2 * zeta * (2 * zeta * delay ** 2 - 1) * torch.exp(-zeta * delay ** 2)) * normalise
            v *= amp
            w[it] = v
    G.waveform = w
    if pmlthick > 0:
        _build_pmls(G, er, mr)
    else:
        G.pmls = []
    _coefficients(G, er, se, mr, adjoint=False)
    torch.cuda.synchronize()
    return G


def _fields(G):
    """The six field arrays (compute.py:499-518), each followed by a zeroed
    tail.  The reference's H kernel reads Ez[i+1] and Ez[j+1] up to
    (ny+1)(nz+1) + (nz+1) floats past the end of the last shot's buffer and
    multiplies them by zero coefficients (src/lib/fields_updates_gpu.cu:65,75);
    with torch's caching allocator that memory can hold NaN from an earlier
    tensor, and NaN * 0 is NaN.  The zeroed tail gives the over-read the value
    the reference's own runs see when it lands on zeros; the kernels and
    their arguments are unchanged."""
    shape = (G.step, int(G.nx) + 1, int(G.ny) + 1, int(G.nz) + 1)
    n = shape[0] * shape[1] * shape[2] * shape[3]
    pad = 2 * shape[2] * shape[3] + 64
    return [torch.zeros(n + pad, device=G.device)[:n].view(shape) for _ in range(6)]  # Ex Ey Ez Hx Hy Hz


def _pml_call(lib, p, which, F, coef, G):
    fn = getattr(lib, "order1_" + p.direction)
    if which == "E":
        P1, P2, RA, RB, RE, RF = p.EPhi1, p.EPhi2, p.ERA, p.ERB, p.ERE, p.ERF
    else:
        P1, P2, RA, RB, RE, RF = p.HPhi1, p.HPhi2, p.HRA, p.HRB, p.HRE, p.HRF
    fn(p.xs, p.xf, p.ys, p.yf, p.zs, p.zf, P1.shape[1], P1.shape[2], P1.shape[3], P2.shape[1], P2.shape[2],
       P2.shape[3], p.thickness, *[fp(x) for x in F], fp(P1), fp(P2), fp(RA), fp(RB), fp(RE), fp(RF),
       float(p.d), fp(coef), int(G.nx) + 1, int(G.ny) + 1, int(G.nz) + 1, G.step)


def forward(G):
    """Forward() of compute.py:542-720.  Returns (rxs (S, 6, nt, nrx), Ez history (nt, S, nx, ny, nz))."""
    L = libs()
    F = _fields(G)
    Ex, Ey, Ez, Hx, Hy, Hz = F
    _alloc_phi(G)
    NX, NY, NZ = int(G.nx) + 1, int(G.ny) + 1, int(G.nz) + 1
    hist = torch.zeros((G.iterations, G.step, int(G.nx), int(G.ny), int(G.nz)), device=G.device)
    rxs = torch.zeros((G.step, 6, G.iterations, G.nrx), device=G.device)
    srcw = torch.zeros((G.nsrc, G.iterations), device=G.device)
    srcw[0, :] = G.waveform
    fu, sr = L["fields_updates_gpu"], L["sourcereceiver"]
    for it in range(G.iterations):
        sr.launch_store_outputs(G.step, G.nrx, it, ip(G.receiver), fp(rxs), *[fp(x) for x in F], NX, NY, NZ, 3, 6,
                                G.iterations)
        fu.h_fields_updates(fp(G.uH0), fp(G.uH1), *[fp(x) for x in F], G.step, NX, NY, NZ)
        for p in G.pmls:
            _pml_call(L["pml_updates_h"], p, "H", F, G.uH4, G)
        fu.e_fields_updates(fp(G.uE0), fp(G.uE1), *[fp(x) for x in F], G.step, NX, NY, NZ)
        for p in G.pmls:
            _pml_call(L["pml_updates_e"], p, "E", F, G.uE4, G)
        sr.update_hertzian_dipole(G.step, it, float(G.dx), float(G.dy), float(G.dz), ip(G.source), float(G.dz),
                                  fp(srcw), fp(Ex), fp(Ey), fp(Ez), fp(G.uE4), NX, NY, NZ, G.nsrc, 2, G.iterations)
        hist[it] = Ez[:, :G.nx, :G.ny, :G.nz]
    torch.cuda.synchronize()
    return rxs, hist


def backward(G, er, se, mr, hist, grad_output, need_er=True, need_se=True, normalize=True):
    """backinitialization() + Backward() of compute.py:945-1180 (no TV term)."""
    L = libs()
    H = Grid()
    for k in ("step", "device", "dx", "dy", "dz", "nx", "ny", "nz", "dt", "iterations", "pmlthickness"):
        setattr(H, k, getattr(G, k))
    H.nrx, H.nsrc = G.nsrc, G.nrx
    H.source = G.receiver
    if any(v > 0 for k, v in H.pmlthickness.items()):
        _build_pmls(H, er, mr)
    else:
        H.pmls = []
    _coefficients(H, er, se, mr, adjoint=True)
    F = _fields(H)
    Ex, Ey, Ez, Hx, Hy, Hz = F
    _alloc_phi(H)
    NX, NY, NZ = int(H.nx) + 1, int(H.ny) + 1, int(H.nz) + 1
    ge = torch.zeros((int(H.nx), int(H.ny), int(H.nz)), device=H.device)
    gs = torch.zeros((int(H.nx), int(H.ny), int(H.nz)), device=H.device)
    g = grad_output.to(H.device).contiguous()
    fu = L["fields_updates_gpu"]
    for it in range(H.iterations - 1, 0, -1):
        L["back"].back_source(H.step, it, float(H.dx), float(H.dy), float(H.dz), ip(H.source), float(H.dz), fp(g),
                              fp(Ex), fp(Ey), fp(Ez), fp(H.uE4), NX, NY, NZ, H.nsrc, 2, H.iterations)
        fu.e_fields_updates(fp(H.uE0), fp(H.uE1), *[fp(x) for x in F], H.step, NX, NY, NZ)
        for p in H.pmls:
            _pml_call(L["pml_updates_e"], p, "E", F, H.uE4, H)
        fu.h_fields_updates(fp(H.uH0), fp(H.uH1), *[fp(x) for x in F], H.step, NX, NY, NZ)
        for p in H.pmls:
            _pml_call(L["pml_updates_h"], p, "H", F, H.uH4, H)
        if need_er:
            ge += torch.sum((hist[it] - hist[it - 1]) * Ez[:, :-1, :-1, :-1], dim=0)
        if need_se:
            gs += torch.sum(hist[it] * Ez[:, :-1, :-1, :-1] * H.dt, dim=0)
    torch.cuda.synchronize()
    if normalize:
        return (ge / ge.norm() if need_er else None), (gs / gs.norm() if need_se else None)
    return (ge if need_er else None), (gs if need_se else None)
