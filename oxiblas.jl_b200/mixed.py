"""mixed_solve on the B200 engine (src/lapack/factorizations.jl:425-427,
src/lapack/extended_lapack.jl:175-226).

    r = mixed_solve(A, b; maxiter=10, rtol=1e-13, precision="fp32", refine="ir")

precision : "fp32" (the reference's default Low = Float32), "bf16" / "fp16"
            (FP32 panels, tensor-core trailing updates with 16-bit operands),
            "bf16x3" (split-BF16 operands, three products accumulated in FP32),
            "fp16x3" (split-FP16 operands, power-of-two scaled, the same three products),
            "fp64" (working-precision factor).
refine    : "ir" (classical, the reference's loop), "gmres" (GMRES-IR),
            "auto" (IR, switching to GMRES-IR when it stagnates).
normwise  : stop on the normwise backward error instead of the componentwise
            one (the reference's metric).
factorization : "lu" (default) or "cholesky" (the Cholesky family: one global
            scale max|a_ij|, the low-precision Cholesky of the lower triangle;
            a factor that is not positive definite falls back to FP64, and
            PosDefException if that fails too).
Returns a dict with the reference's NamedTuple fields (x, converged,
iterations, residual, backward_error, metric, low_type, fallback, finite,
reason) plus backward_error_normwise, gmres_iterations, factor_ms, refine_ms.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import (ArgumentError, DimensionMismatch, Handle, SingularException, OPT_STOP_NORMWISE,
                   OXI_ENONFINITE, OXI_ENOTCONVERGED, OXI_ESINGULAR, OXI_OK)

OXI_ENOTPOSDEF = 10
from .lu import colmajor_copy, _as_tensor

PREC = {"fp32": 0, "bf16": 1, "fp16": 2, "fp64": 3, "bf16x3": 4, "fp16x3": 5}
REFINE = {"ir": 0, "gmres": 1, "auto": 2}
REASONS = ("converged", "iteration_limit", "working_factor_fallback", "nonfinite_iteration")


class RefineReport(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("gmres_iterations", ctypes.c_int64),
                ("backward_error", ctypes.c_double), ("backward_error_normwise", ctypes.c_double),
                ("residual_norm", ctypes.c_double), ("factor_ms", ctypes.c_double),
                ("refine_ms", ctypes.c_double), ("info", ctypes.c_int64),
                ("converged", ctypes.c_int32), ("fallback", ctypes.c_int32),
                ("refine_used", ctypes.c_int32), ("reason", ctypes.c_int32),
                ("low_type", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def mixed_solve_device(Acm: torch.Tensor, Bcm: torch.Tensor, Xcm: torch.Tensor, n: int, nrhs: int,
                       maxiter=10, rtol=1e-13, precision="fp32", refine="ir", normwise=False,
                       factorization="lu"):
    """Device-resident call: Acm (n, n) contiguous is the column-major A, Bcm and
    Xcm (nrhs, n) contiguous are column-major B and X.  Returns (status, report)."""
    h = Handle.get()
    rep = RefineReport()
    old = h.get_option(OPT_STOP_NORMWISE)
    h.set_option(OPT_STOP_NORMWISE, 1 if normwise else 0)
    try:
        fn = h.lib.oxi_dposv_mixed if factorization == "cholesky" else h.lib.oxi_dgesv_mixed
        st = fn(h.ptr, PREC[precision], REFINE[refine], n, nrhs,
                                   ctypes.c_void_p(Acm.data_ptr()), max(1, n),
                                   ctypes.c_void_p(Bcm.data_ptr()), max(1, n),
                                   ctypes.c_void_p(Xcm.data_ptr()), max(1, n), int(maxiter),
                                   float(rtol), ctypes.byref(rep))
    finally:
        h.set_option(OPT_STOP_NORMWISE, old)
    return st, rep


def mixed_solve(A, b, *, maxiter: int = 10, rtol: float = 1e-13, precision: str = "fp32",
                refine: str = "ir", normwise: bool = False, fallback: bool = True,
                factorization: str = "lu"):
    if factorization not in ("lu", "cholesky"):
        raise ArgumentError("unknown mixed factorization")
    if precision not in PREC:
        raise ArgumentError("low precision type must be one of " + ", ".join(PREC))
    if refine not in REFINE:
        raise ArgumentError("refine must be one of " + ", ".join(REFINE))
    if maxiter < 0 or not np.isfinite(rtol) or rtol < 0:
        raise ArgumentError("invalid mixed solve options")
    At = _as_tensor(A)
    bt = _as_tensor(b)
    if At.ndim != 2 or At.shape[0] != At.shape[1]:
        raise DimensionMismatch("mixed factorization dimensions differ")
    n = At.shape[0]
    vec = bt.ndim == 1
    B2 = bt.reshape(n, -1) if bt.shape[0] == n else None
    if B2 is None:
        raise DimensionMismatch("right-hand side rows differ")
    nrhs = B2.shape[1]
    if n == 0 or nrhs == 0:
        x = torch.zeros_like(bt, dtype=torch.float64)
        return dict(x=x, converged=True, iterations=0, residual=0.0, backward_error=0.0,
                    backward_error_normwise=0.0, metric="componentwise_backward_error",
                    low_type=precision, fallback=False, finite=True, reason="converged",
                    gmres_iterations=0, factor_ms=0.0, refine_ms=0.0)
    Acm = colmajor_copy(At, torch.float64)
    Bcm = colmajor_copy(B2, torch.float64)
    Xcm = torch.zeros_like(Bcm)
    reps = []
    for k0 in range(0, nrhs, 16):
        k1 = min(nrhs, k0 + 16)
        st, rep = mixed_solve_device(Acm, Bcm[k0:k1], Xcm[k0:k1], n, k1 - k0, maxiter, rtol,
                                     precision, refine, normwise, factorization)
        h = Handle.get()
        if st == OXI_ENONFINITE:
            raise ArgumentError("finite mixed input required")
        if st == OXI_ESINGULAR:
            raise SingularException(rep.info)
        if st == OXI_ENOTPOSDEF:
            from .cholesky import PosDefException
            raise PosDefException(rep.info)
        if st not in (OXI_OK, OXI_ENOTCONVERGED):
            h.check(st)
        if rep.fallback and not fallback:
            if factorization == "cholesky":
                from .cholesky import PosDefException
                raise PosDefException(rep.info)
            raise SingularException(rep.info)
        reps.append(rep)
    X = Xcm.t()
    x = X[:, 0].clone() if vec else X.clone()
    worst = max(reps, key=lambda r: r.backward_error)
    err = max(r.backward_error for r in reps)
    finite = bool(torch.isfinite(X).all().item()) and np.isfinite(err)
    return dict(x=x, converged=all(r.converged for r in reps),
                iterations=max(r.iterations for r in reps),
                residual=float(np.sqrt(sum(r.residual_norm ** 2 for r in reps))),
                backward_error=err,
                backward_error_normwise=max(r.backward_error_normwise for r in reps),
                metric="componentwise_backward_error", low_type=precision,
                fallback=any(r.fallback for r in reps), finite=finite, factorization=factorization,
                reason=REASONS[worst.reason] if finite else "nonfinite_iteration",
                gmres_iterations=sum(r.gmres_iterations for r in reps),
                refine_used=("ir", "gmres", "auto")[worst.refine_used],
                factor_ms=sum(r.factor_ms for r in reps), refine_ms=sum(r.refine_ms for r in reps))


def equilibrate(A, radix: bool = True):
    """equilibrate(A; radix=true) (src/lapack/dense_utilities.jl:191-213) on the
    GPU: returns dict(matrix, row_scale, column_scale) with
    matrix = A ./ row_scale ./ column_scale', the scales powers of two."""
    if not radix:
        raise ArgumentError("only the radix (power-of-two) equilibration runs on the GPU engine")
    At = _as_tensor(A)
    if At.ndim != 2:
        raise DimensionMismatch("a matrix is required")
    m, n = At.shape
    Acm = colmajor_copy(At, torch.float64)  # (n, m) storage = column-major A
    Ecm = torch.empty_like(Acm)
    rows = torch.ones(m, dtype=torch.float64, device=Acm.device)
    cols = torch.ones(n, dtype=torch.float64, device=Acm.device)
    h = Handle.get()
    st = h.lib.oxi_dequilibrate(h.ptr, m, n, ctypes.c_void_p(Acm.data_ptr()), max(1, m),
                                ctypes.c_void_p(rows.data_ptr()), ctypes.c_void_p(cols.data_ptr()),
                                ctypes.c_void_p(Ecm.data_ptr()), max(1, m))
    if st == OXI_ENONFINITE:
        raise ArgumentError("finite input required")
    h.check(st)
    return dict(matrix=Ecm.t(), row_scale=rows, column_scale=cols)


def gemm_update_lowp(C: torch.Tensor, A: torch.Tensor, B: torch.Tensor, precision="bf16"):
    """C <- C - A @ B with A, B rounded to 16 bits and FP32 accumulation: the
    mixed path's trailing-update kernel (tcgen05) on float32 CUDA tensors."""
    for X in (C, A, B):
        if X.dtype != torch.float32 or not X.is_cuda or X.stride(1) != 1:
            raise ArgumentError("float32 CUDA tensors with unit inner stride required")
    m, k = A.shape
    n = B.shape[1]
    h = Handle.get()
    st = h.lib.oxi_sgemm_update_lowp(h.ptr, PREC[precision], n, m, k, ctypes.c_void_p(C.data_ptr()),
                                     C.stride(0), ctypes.c_void_p(B.data_ptr()), B.stride(0),
                                     ctypes.c_void_p(A.data_ptr()), A.stride(0))
    h.check(st)
    return C
