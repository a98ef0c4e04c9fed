"""Drop-in ``total_variation`` (reference src/tv.py:135-217).

ADMM total-variation denoising of a 2-D model, as used by the reference's
gradient (src/compute.py:916-933: grad += 0.01 * 2 * (m - TV(m))).  The model
is scaled by 1/(max + 1e-6), embedded in a zero border of one cell, and
iterated up to ``num_iter`` times:

    X  <- (lambda*rho*N4(X) + [Y + lambda*rho*Dt(Z) - lambda*Dt(U)]) / (1 + 4 lambda rho)
    Z  <- shrink(U/rho + D(X), 1/rho)            (soft threshold)
    U  <- U + rho*(D(X) - Z)

with D the periodic forward difference along each axis, Dt its adjoint and
N4 the sum of the four neighbours; it stops early when ||X - X_prev|| < tol.
The arguments and in-place squeeze of the input follow the reference.
"""
from __future__ import annotations

import torch


def _dt(z: torch.Tensor, dim: int) -> torch.Tensor:
    """Adjoint of the periodic backward difference: z[k] - z[k+1] (wrapping)."""
    return z - torch.roll(z, -1, dims=dim)


def _d(x: torch.Tensor, dim: int) -> torch.Tensor:
    """Periodic backward difference: x[k] - x[k-1] (wrapping)."""
    return x - torch.roll(x, 1, dims=dim)


def total_variation(data, lamda=0.02, rho=1.0, num_iter=500, tol=1e-5, capturable=False):
    """float32 CUDA models run the whole ADMM solve as one kernel
    (fg_total_variation, libfastgpr.so); other tensors (CPU, float64) take
    the tensor arithmetic below, which is the reference's own.
    capturable=True (not in the reference): the kernel is only enqueued, with
    no wait for its iteration count, so the call may be captured in a CUDA
    graph."""
    data.squeeze_(-1)
    if data.is_cuda and data.dtype == torch.float32 and data.dim() == 2:
        from . import _native
        out, _ = _native.total_variation(data, lamda, rho, num_iter, tol, wait=not capturable)
        return out.unsqueeze(-1)
    return _total_variation_tensor(data, lamda, rho, num_iter, tol)


def _total_variation_tensor(data, lamda=0.02, rho=1.0, num_iter=500, tol=1e-5):
    data_max = data.max()
    scaled = data / (data_max + 1e-6)
    M, N = scaled.shape
    X = torch.zeros((M + 2, N + 2), device=data.device)
    X[1:-1, 1:-1] = scaled
    Y = X.clone()
    Zx = torch.zeros_like(X)
    Zy = torch.zeros_like(X)
    Ux = torch.zeros_like(X)
    Uy = torch.zeros_like(X)
    lr = lamda * rho
    for _ in range(num_iter):
        X_prev = X.clone()
        rhs = Y + lr * (_dt(Zx, 1) + _dt(Zy, 0)) - lamda * (_dt(Ux, 1) + _dt(Uy, 0))
        nsum = X[0:-2, 1:-1] + X[1:-1, 0:-2] + X[1:-1, 2:] + X[2:, 1:-1]
        X[1:-1, 1:-1] = (nsum * lamda * rho + rhs[1:-1, 1:-1]) / (1 + 4 * lamda * rho)
        dxX = _d(X, 1)
        dyX = _d(X, 0)
        tx = (Ux + rho * dxX) / rho
        Zx = torch.sign(tx) * torch.clamp(torch.abs(tx) - 1 / rho, min=0)
        ty = (Uy + rho * dyX) / rho
        Zy = torch.sign(ty) * torch.clamp(torch.abs(ty) - 1 / rho, min=0)
        Ux += rho * (dxX - Zx)
        Uy += rho * (dyX - Zy)
        if torch.norm(X - X_prev) < tol:
            break
    return (X[1:-1, 1:-1] * data_max).unsqueeze(-1)
