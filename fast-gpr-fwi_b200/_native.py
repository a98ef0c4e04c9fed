"""ctypes binding of libfastgpr.so (the C ABI in include/fastgpr.h).

The library is built in-tree (``build.py``) and loaded from ``_lib/``.  There
is no fallback: if the library is missing or no CUDA device is present, every
solve raises.  Setting FASTGPR_CHECKED=1 loads the bounds-checked build
(``libfastgpr_checked.so``), whose kernels test every global access and
record a violation instead of touching memory out of range.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "_lib")

FG_OK = 0
FG_ERR_INVALID = 1
FG_ERR_CUDA = 2
FG_ERR_WORKSPACE = 3
FG_ERR_TIMEOUT = 4

# Every entry point include/fastgpr.h declares (checked by the tests).
EXPORTS = (
    "fg_plan_create", "fg_plan_destroy", "fg_plan_hist_shape", "fg_plan_workspace_bytes", "fg_plan_bind",
    "fg_coefficients", "fg_forward", "fg_adjoint_reference", "fg_plan_check", "fg_last_error",
    "fg_forward_static", "fg_tv_workspace_bytes", "fg_total_variation",
    "fg_plan_checkpoint_bytes", "fg_forward_checkpointed", "fg_adjoint_reference_checkpointed",
    "fg_fir_causal", "fg_adjoint_reference_l1", "fg_adjoint_exact",
    "fg_forward_batch", "fg_adjoint_reference_batch", "fg_plan_set_profile", "fg_plan_shape",
)

BATCH_MAX = 8   # FG_BATCH_MAX


class FgProblem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("shots", ctypes.c_int32),
        ("nt", ctypes.c_int32), ("th", ctypes.c_int32),
        ("dx", ctypes.c_float), ("dt", ctypes.c_float),
        ("nsrc", ctypes.c_int32), ("nrx", ctypes.c_int32),
        ("src", ctypes.POINTER(ctypes.c_int32)), ("rx", ctypes.POINTER(ctypes.c_int32)),
        ("srcw", ctypes.POINTER(ctypes.c_float)), ("pml", ctypes.POINTER(ctypes.c_float)),
    ]


class FgTuning(ctypes.Structure):
    _fields_ = [
        ("lanes", ctypes.c_int32), ("cells_per_thread", ctypes.c_int32), ("rows_per_tile", ctypes.c_int32),
        ("warps_per_block", ctypes.c_int32), ("stages", ctypes.c_int32), ("kernel", ctypes.c_int32),
        ("adj_kernel", ctypes.c_int32), ("adj_rows_per_tile", ctypes.c_int32),
        ("adj_warps_per_block", ctypes.c_int32), ("adj_stages", ctypes.c_int32),
        ("adj_cells_per_thread", ctypes.c_int32), ("prefetch", ctypes.c_int32), ("interior", ctypes.c_int32),
        ("persistent", ctypes.c_int32), ("slab", ctypes.c_int32),
    ]

    KEYS = ("lanes", "cells_per_thread", "rows_per_tile", "warps_per_block", "stages", "kernel",
            "adj_kernel", "adj_rows_per_tile", "adj_warps_per_block", "adj_stages", "adj_cells_per_thread",
            "prefetch", "interior", "persistent", "slab")


class FastGprError(RuntimeError):
    """A libfastgpr call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__("libfastgpr error %d: %s" % (code, msg))
        self.code = code


_lib: Optional[ctypes.CDLL] = None


def checked_build() -> bool:
    return os.environ.get("FASTGPR_CHECKED", "0") not in ("", "0")


def library_path(checked: Optional[bool] = None) -> str:
    if checked is None:
        checked = checked_build()
    name = "libfastgpr_checked.so" if checked else "libfastgpr.so"
    return os.path.join(LIB_DIR, name)


def lib() -> ctypes.CDLL:
    """Load libfastgpr.so once and declare the signatures."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise FastGprError(FG_ERR_INVALID, "%s is not built; run build.py (or __graft_entry__.build())" % path)
    L = ctypes.CDLL(path)
    vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    L.fg_plan_create.argtypes = [ctypes.POINTER(FgProblem), ctypes.POINTER(FgTuning), ctypes.POINTER(vp)]
    L.fg_plan_create.restype = ctypes.c_int
    L.fg_plan_destroy.argtypes = [vp]
    L.fg_plan_destroy.restype = ctypes.c_int
    L.fg_plan_hist_shape.argtypes = [vp, ctypes.POINTER(i64)]
    L.fg_plan_hist_shape.restype = ctypes.c_int
    L.fg_plan_workspace_bytes.argtypes = [vp]
    L.fg_plan_workspace_bytes.restype = i64
    L.fg_plan_shape.argtypes = [vp, ctypes.POINTER(i32)]
    L.fg_plan_shape.restype = ctypes.c_int
    L.fg_plan_bind.argtypes = [vp, vp, i64, vp]
    L.fg_plan_bind.restype = ctypes.c_int
    L.fg_coefficients.argtypes = [vp, vp, vp, i32, i32, f32, f32, i32, vp, i32, vp]
    L.fg_coefficients.restype = ctypes.c_int
    L.fg_forward.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.fg_forward.restype = ctypes.c_int
    L.fg_adjoint_reference.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp]
    L.fg_adjoint_reference.restype = ctypes.c_int
    L.fg_forward_static.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.fg_forward_static.restype = ctypes.c_int
    L.fg_plan_checkpoint_bytes.argtypes = [vp, i32]
    L.fg_plan_checkpoint_bytes.restype = i64
    L.fg_forward_checkpointed.argtypes = [vp, vp, vp, vp, vp, vp, i64, i32, vp]
    L.fg_forward_checkpointed.restype = ctypes.c_int
    L.fg_adjoint_reference_checkpointed.argtypes = [vp, vp, vp, vp, vp, i64, i32, vp, vp, vp, vp, i32, vp, vp]
    L.fg_adjoint_reference_checkpointed.restype = ctypes.c_int
    L.fg_adjoint_reference_l1.argtypes = [vp, vp, vp, vp, vp, vp, vp, f32, vp, vp, i32, vp, vp]
    L.fg_adjoint_reference_l1.restype = ctypes.c_int
    L.fg_adjoint_exact.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.fg_adjoint_exact.restype = ctypes.c_int
    L.fg_plan_set_profile.argtypes = [vp, vp, vp]
    L.fg_plan_set_profile.restype = ctypes.c_int
    L.fg_forward_batch.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp]
    L.fg_forward_batch.restype = ctypes.c_int
    L.fg_adjoint_reference_batch.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, i32, vp]
    L.fg_adjoint_reference_batch.restype = ctypes.c_int
    L.fg_fir_causal.argtypes = [vp, i64, i32, i32, vp, i32, vp, vp]
    L.fg_fir_causal.restype = ctypes.c_int
    L.fg_tv_workspace_bytes.argtypes = [i32, i32]
    L.fg_tv_workspace_bytes.restype = i64
    L.fg_total_variation.argtypes = [vp, i32, i32, ctypes.c_double, ctypes.c_double, i32, ctypes.c_double, vp, vp,
                                     i64, ctypes.POINTER(i32), vp]
    L.fg_total_variation.restype = ctypes.c_int
    L.fg_plan_check.argtypes = [vp, vp]
    L.fg_plan_check.restype = ctypes.c_int
    L.fg_last_error.argtypes = []
    L.fg_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != FG_OK:
        raise FastGprError(rc, lib().fg_last_error().decode(errors="replace"))


def ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class Plan:
    """A planned solve geometry with its bound device workspace."""

    def __init__(self, nx, ny, shots, nt, th, dx32, dt32, src: np.ndarray, rx: np.ndarray,
                 srcw: np.ndarray, pml: Optional[np.ndarray], device, tuning=None, bind: bool = True):
        L = lib()
        self.device = torch.device(device)
        self.nx, self.ny, self.shots, self.nt, self.th = int(nx), int(ny), int(shots), int(nt), int(th)
        self._src = np.ascontiguousarray(src, dtype=np.int32)
        self._rx = np.ascontiguousarray(rx, dtype=np.int32)
        self._srcw = np.ascontiguousarray(srcw, dtype=np.float32)
        self._pml = None if pml is None else np.ascontiguousarray(pml, dtype=np.float32)
        self.nsrc = self._src.shape[1] if self._src.ndim == 3 else 0
        self.nrx = self._rx.shape[1] if self._rx.ndim == 3 else 0
        prob = FgProblem()
        prob.nx, prob.ny, prob.shots, prob.nt, prob.th = self.nx, self.ny, self.shots, self.nt, self.th
        prob.dx, prob.dt = float(dx32), float(dt32)
        prob.nsrc, prob.nrx = self.nsrc, self.nrx
        prob.src = self._src.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        prob.rx = self._rx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        prob.srcw = self._srcw.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        prob.pml = (self._pml.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
                    if self._pml is not None else ctypes.POINTER(ctypes.c_float)())
        tune = None
        if tuning is not None:
            unknown = set(tuning) - set(FgTuning.KEYS)
            if unknown:
                raise ValueError("unknown tuning keys: %s" % sorted(unknown))
            tune = FgTuning(*[int(tuning.get(k, 0)) for k in FgTuning.KEYS])
        handle = ctypes.c_void_p()
        check(L.fg_plan_create(ctypes.byref(prob), ctypes.byref(tune) if tune is not None else None,
                               ctypes.byref(handle)))
        self._h = handle
        shape = (ctypes.c_int64 * 5)()
        check(L.fg_plan_hist_shape(handle, shape))
        self.hist_shape = tuple(int(v) for v in shape)   # (nt, groups, nx, pitch, slots)
        self.hist_floats = int(np.prod(self.hist_shape))
        self.workspace_bytes = int(L.fg_plan_workspace_bytes(handle))
        self.workspace = None
        if bind:
            self.bind()

    def bind(self):
        """Allocate the device workspace and upload the plan's tables."""
        if self.workspace is None:
            self.workspace = torch.empty(self.workspace_bytes, dtype=torch.uint8, device=self.device)
            check(lib().fg_plan_bind(self._h, self.workspace.data_ptr(), self.workspace_bytes,
                                     stream_handle(self.device)))

    SHAPE_KEYS = ("kernel", "lanes", "cells_per_thread", "rows_per_tile", "warps_per_block", "stages",
                  "interior_split", "slab_blocks_per_sm", "persistent")

    def shape(self) -> dict:
        """The launch shapes the plan chose (fg_plan_shape), host-side:
        {'forward': {...}, 'adjoint': {...}} with the keys of SHAPE_KEYS."""
        out = (ctypes.c_int32 * 18)()
        check(lib().fg_plan_shape(self._h, out))
        n = len(self.SHAPE_KEYS)
        return {d: dict(zip(self.SHAPE_KEYS, (int(v) for v in out[k * n:(k + 1) * n])))
                for k, d in enumerate(("forward", "adjoint"))}

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.fg_plan_destroy(h)
            self._h = None

    def new_hist(self) -> torch.Tensor:
        """An uninitialised Ez history buffer for this plan (flat float32)."""
        return torch.empty(self.hist_floats, dtype=torch.float32, device=self.device)

    def hist_view(self, hist: torch.Tensor) -> torch.Tensor:
        """History as (nt, shots, nx, ny) (a copy when shots share cells)."""
        nt, groups, nx, pitch, slots = self.hist_shape
        h = hist.view(nt, groups, nx, pitch, slots).permute(0, 1, 4, 2, 3).reshape(nt, groups * slots, nx, pitch)
        return h[:, :self.shots, :, :self.ny]

    def set_profile(self, pml: np.ndarray):
        """fg_plan_set_profile: a new CPML profile (8 * th floats), same tables and buffers."""
        self._pml = np.ascontiguousarray(pml, dtype=np.float32)
        if self._pml.size != 8 * self.th:
            raise ValueError("profile must hold 8 * th = %d floats" % (8 * self.th))
        check(lib().fg_plan_set_profile(self._h, self._pml.ctypes.data, stream_handle(self.device)))

    def device_check(self):
        """Synchronise and raise if a kernel recorded a device-side error."""
        check(lib().fg_plan_check(self._h, stream_handle(self.device)))

    def forward(self, er32, se32, mr32, traces, hist):
        check(lib().fg_forward(self._h, ptr(er32), ptr(se32), ptr(mr32), ptr(traces), ptr(hist),
                               stream_handle(self.device)))
        if checked_build():
            self.device_check()

    def adjoint_reference(self, er32, se32, mr32, hist, resid, grad_eps, grad_sig, normalize=True, norms=None):
        check(lib().fg_adjoint_reference(self._h, ptr(er32), ptr(se32), ptr(mr32), ptr(hist), ptr(resid),
                                         ptr(grad_eps), ptr(grad_sig), 1 if normalize else 0, ptr(norms),
                                         stream_handle(self.device)))
        if checked_build():
            self.device_check()

    def adjoint_reference_l1(self, er32, se32, mr32, hist, traces, observed, scale, grad_eps, grad_sig,
                             normalize=True, norms=None):
        """Adjoint of the L1 misfit scale * sum |traces - observed|, injected on the fly."""
        check(lib().fg_adjoint_reference_l1(self._h, ptr(er32), ptr(se32), ptr(mr32), ptr(hist), ptr(traces),
                                            ptr(observed), float(scale), ptr(grad_eps), ptr(grad_sig),
                                            1 if normalize else 0, ptr(norms), stream_handle(self.device)))
        if checked_build():
            self.device_check()

    def adjoint_exact(self, er32, se32, mr32, hist, weights, grad_eps, grad_sig):
        """Exact gradient of sum(weights * traces) (fg_adjoint_exact), not normalised."""
        check(lib().fg_adjoint_exact(self._h, ptr(er32), ptr(se32), ptr(mr32), ptr(hist), ptr(weights),
                                     ptr(grad_eps), ptr(grad_sig), stream_handle(self.device)))
        if checked_build():
            self.device_check()

    # checkpointed solve (fg_forward_checkpointed / fg_adjoint_reference_checkpointed)
    def checkpoint_bytes(self, interval: int) -> int:
        return int(lib().fg_plan_checkpoint_bytes(self._h, int(interval)))

    def new_checkpoints(self, interval: int) -> torch.Tensor:
        """Checkpoint buffer for `interval` (at least 16 bytes, so it has an address)."""
        return torch.empty(max(16, self.checkpoint_bytes(interval)), dtype=torch.uint8, device=self.device)

    def new_segment(self, interval: int) -> torch.Tensor:
        """History buffer of one segment of `interval` steps (flat float32)."""
        return torch.empty(min(int(interval), self.nt) * (self.hist_floats // self.nt), dtype=torch.float32,
                           device=self.device)

    def forward_checkpointed(self, er32, se32, mr32, traces, ckpt, interval):
        check(lib().fg_forward_checkpointed(self._h, ptr(er32), ptr(se32), ptr(mr32), ptr(traces), ptr(ckpt),
                                            ckpt.numel() * ckpt.element_size(), int(interval),
                                            stream_handle(self.device)))
        if checked_build():
            self.device_check()

    def adjoint_reference_checkpointed(self, er32, se32, mr32, ckpt, interval, segment, resid, grad_eps, grad_sig,
                                       normalize=True, norms=None):
        if segment.numel() < min(int(interval), self.nt) * (self.hist_floats // self.nt):
            raise ValueError("segment buffer too small for interval %d" % interval)
        check(lib().fg_adjoint_reference_checkpointed(
            self._h, ptr(er32), ptr(se32), ptr(mr32), ptr(ckpt), ckpt.numel() * ckpt.element_size(), int(interval),
            ptr(segment), ptr(resid), ptr(grad_eps), ptr(grad_sig), 1 if normalize else 0, ptr(norms),
            stream_handle(self.device)))
        if checked_build():
            self.device_check()


def _ptrs(ts) -> ctypes.Array:
    return (ctypes.c_void_p * len(ts))(*[ptr(t) for t in ts])


def forward_batch(plans, er32, se32, mr32, traces, hists):
    """fg_forward_batch: the forward solves of several plans in one launch.

    Every argument is a sequence with one entry per plan (hists entries may be
    None); all plans on one device.
    """
    n = len(plans)
    hs = (ctypes.c_void_p * n)(*[p.handle for p in plans])
    check(lib().fg_forward_batch(hs, n, _ptrs(er32), _ptrs(se32), _ptrs(mr32), _ptrs(traces), _ptrs(hists),
                                 stream_handle(plans[0].device)))
    if checked_build():
        for p in plans:
            p.device_check()


def adjoint_reference_batch(plans, er32, se32, mr32, hists, resids, grad_eps, grad_sig, normalize=True):
    """fg_adjoint_reference_batch: the adjoint solves of several plans in one launch."""
    n = len(plans)
    hs = (ctypes.c_void_p * n)(*[p.handle for p in plans])
    check(lib().fg_adjoint_reference_batch(hs, n, _ptrs(er32), _ptrs(se32), _ptrs(mr32), _ptrs(hists),
                                           _ptrs(resids), _ptrs(grad_eps), _ptrs(grad_sig),
                                           1 if normalize else 0, stream_handle(plans[0].device)))
    if checked_build():
        for p in plans:
            p.device_check()


def coefficients(er32, se32, mr32, dt32, dx32, adjoint, pitch=None):
    """fg_coefficients into a fresh (5, nx+1, pitch) tensor."""
    nx, ny = er32.shape
    if pitch is None:
        pitch = (ny + 1 + 31) // 32 * 32
    out = torch.empty((5, nx + 1, pitch), dtype=torch.float32, device=er32.device)
    check(lib().fg_coefficients(ptr(er32), ptr(se32), ptr(mr32), nx, ny, float(dt32), float(dx32),
                                1 if adjoint else 0, ptr(out), pitch, stream_handle(er32.device)))
    return out


def total_variation(data: torch.Tensor, lamda: float, rho: float, num_iter: int, tol: float, wait: bool = True):
    """fg_total_variation on a 2-D float32 CUDA tensor: (denoised copy,
    iterations).  wait=False only enqueues (capturable in a CUDA graph; the
    iteration count is then None and a barrier time-out is not reported)."""
    if data.dim() != 2 or data.dtype != torch.float32 or not data.is_cuda:
        raise ValueError("total_variation kernel: needs a 2-D float32 CUDA tensor")
    L = lib()
    d = data.contiguous()
    M, N = d.shape
    out = torch.empty_like(d)
    ws = torch.empty(int(L.fg_tv_workspace_bytes(M, N)), dtype=torch.uint8, device=d.device)
    iters = ctypes.c_int32(0)
    with torch.cuda.device(d.device):
        stream = torch.cuda.current_stream(d.device).cuda_stream
        check(L.fg_total_variation(d.data_ptr(), M, N, float(lamda), float(rho), int(num_iter), float(tol),
                                   out.data_ptr(), ws.data_ptr(), ws.numel(), ctypes.byref(iters) if wait else None,
                                   stream))
    return out, int(iters.value) if wait else None


def fir_causal(x: torch.Tensor, taps: torch.Tensor) -> torch.Tensor:
    """fg_fir_causal on a float32 CUDA tensor of shape (batch, T, R); taps (k,)."""
    if x.dim() != 3 or x.dtype != torch.float32 or not x.is_cuda:
        raise ValueError("fir kernel: needs a 3-D float32 CUDA tensor (batch, T, R)")
    L = lib()
    xc = x.contiguous()
    h = taps.to(device=x.device, dtype=torch.float32).contiguous()
    out = torch.empty_like(xc)
    b, T, R = xc.shape
    with torch.cuda.device(x.device):
        check(L.fg_fir_causal(xc.data_ptr(), b, T, R, h.data_ptr(), h.numel(), out.data_ptr(),
                              torch.cuda.current_stream(x.device).cuda_stream))
    return out
