"""Reverse-mode rule of x = A \\ b on the B200 engine.

    bbar, Abar = lu_adjoint(F, x, xbar)     the rrule's pullback with F reused
    x = solve(A, b)                          differentiable A \\ b (torch.autograd)

The reference has no differentiation rule; this is the pullback a
ChainRulesCore ``rrule(::typeof(\\), A, b)`` returns, built on its transposed
solve (``ldiv!(transpose(F), B)``, src/api/linalg_api.jl:176-184, and
``solve_transposed``, src/lapack/expert_refinement.jl:2-23):
lambda = A^-T xbar, bbar = lambda, Abar = -lambda x^T.  Both steps run in
liboxiblas_b200.so (``oxi_dlu_adjoint``).
"""
from __future__ import annotations

import ctypes

import torch

from ._lib import ArgumentError, DimensionMismatch, Handle
from .lu import LU, _as_tensor, lu


def _cm(t: torch.Tensor, n: int, dev) -> torch.Tensor:
    """(k, n) contiguous float64 tensor whose memory is the n x k column-major matrix."""
    t = _as_tensor(t).to(device=dev, dtype=torch.float64)
    if t.shape[0] != n:
        raise DimensionMismatch(f"factorization has {n} rows, vector has {t.shape[0]}")
    return t.reshape(n, -1).t().contiguous()


def lu_adjoint(F: LU, x, xbar):
    """(bbar, Abar) for x = A \\ b and upstream gradient xbar = dL/dx.

    F: the float64 factorization of A (lu(A)); x, xbar: (n,) or (n, k).
    Returns bbar with xbar's shape and Abar (n, n), both float64 on F's device.
    """
    if not isinstance(F, LU) or F.dtype != torch.float64:
        raise ArgumentError("lu_adjoint needs a float64 LU factorization")
    F._ready()
    n = F.shape[0]
    dev = F._buf.device
    shape = tuple(_as_tensor(xbar).shape)
    X = _cm(x, n, dev)
    Xb = _cm(xbar, n, dev)
    if X.shape != Xb.shape:
        raise DimensionMismatch("x and xbar differ in shape")
    k = X.shape[0]
    Bb = torch.empty_like(Xb)
    Abuf = torch.empty((n, n), dtype=torch.float64, device=dev)  # memory = Abar column-major
    h = Handle.get()
    ld = max(1, n)
    st = h.lib.oxi_dlu_adjoint(h.ptr, n, k, ctypes.c_void_p(F._buf.data_ptr()), F._lda,
                               ctypes.c_void_p(F._ipiv.data_ptr()), ctypes.c_void_p(X.data_ptr()), ld,
                               ctypes.c_void_p(Xb.data_ptr()), ld, ctypes.c_void_p(Bb.data_ptr()), ld,
                               ctypes.c_void_p(Abuf.data_ptr()), ld)
    h.check(st)
    return Bb.t().reshape(shape), Abuf.t()


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A, b):
        F = lu(A.detach().to(torch.float64))
        x = F.solve(b.detach().to(torch.float64))
        ctx.F = F
        ctx.devs = (A.device, A.dtype, b.device, b.dtype)
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, xbar):
        (x,) = ctx.saved_tensors
        bbar, Abar = lu_adjoint(ctx.F, x, xbar)
        adev, adt, bdev, bdt = ctx.devs
        return Abar.to(device=adev, dtype=adt), bbar.to(device=bdev, dtype=bdt)


def solve(A: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """x = A \\ b (float64, on the GPU) with the hand-written pullback for autograd."""
    return _Solve.apply(A, b)
