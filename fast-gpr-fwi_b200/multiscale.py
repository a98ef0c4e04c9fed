"""Drop-in ``design_fir_filter`` / ``apply_filter`` (reference src/multiscale.py).

A Hamming-windowed sinc low-pass with ``int(fs / cutoff)`` taps, applied
causally: the series is reflect-padded by ``numtaps - 1`` samples on the left
and cross-correlated with the taps, so output sample t sees input samples
t - numtaps + 1 .. t.  Accepts a 1-D series or (step, iterations, nrx)
receiver traces (time on axis 1), as the reference does (src/multiscale.py:19-53).

The tap design follows src/multiscale.py:4-17 operation for operation in
float32, including its centre-tap assignment at index (numtaps - 1) // 2,
which for an even tap count lands half a sample left of the window centre.
"""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F


def design_fir_filter(cutoff: float, fs: float, numtaps: int) -> torch.Tensor:
    """Normalised Hamming-windowed sinc taps (float32, CPU)."""
    n = torch.arange(numtaps, dtype=torch.float32)
    half = (numtaps - 1) / 2
    window = 0.54 - 0.46 * torch.cos(2 * math.pi * n / (numtaps - 1))
    offset = n - half
    taps = torch.sin(2 * math.pi * (cutoff / fs) * offset) / (math.pi * offset)
    taps[(numtaps - 1) // 2] = 2 * cutoff / fs
    h = window * taps
    return h / h.sum()


def _fir_causal(series: torch.Tensor, taps: torch.Tensor) -> torch.Tensor:
    """series: (B, 1, T) -> (B, 1, T) causal FIR with left reflect padding."""
    k = taps.numel()
    padded = F.pad(series, (k - 1, 0), mode="reflect")
    return F.conv1d(padded, taps.view(1, 1, -1), padding=0)


def apply_filter(data: torch.Tensor, fs: float, cutoff: float) -> torch.Tensor:
    """Low-pass ``data`` (1-D, or (step, iterations, nrx)) at ``cutoff`` Hz.

    float32 CUDA data runs on fg_fir_causal (libfastgpr.so), which filters
    the (step, iterations, nrx) layout along axis 1 directly; other tensors
    take the reference's tensor arithmetic below."""
    numtaps = int(1 * (fs / cutoff))
    taps = design_fir_filter(cutoff, fs, numtaps)
    if data.is_cuda and data.dtype == torch.float32 and data.ndim in (1, 3):
        from . import _native
        if data.ndim == 1:
            return _native.fir_causal(data.view(1, -1, 1), taps).view(-1)
        return _native.fir_causal(data, taps)
    taps = taps.to(data.device)
    if data.ndim == 1:
        return _fir_causal(data.view(1, 1, -1), taps).view(-1)
    if data.ndim == 3:
        step, iterations, nrx = data.shape
        series = data.permute(0, 2, 1).reshape(-1, 1, iterations)
        out = _fir_causal(series, taps)
        return out.view(step, nrx, iterations).permute(0, 2, 1)
    raise ValueError("unsupported data dimension %d: expected a 1-D or 3-D tensor" % data.ndim)
