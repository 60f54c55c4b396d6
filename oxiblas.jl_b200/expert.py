"""Expert solves, the condition estimate, inv and factorize on the B200 engine.

    expert_solve(A, b; maxiter=8, rtol=8eps, equilibrate=True)
        src/lapack/advanced_factorizations.jl:591-645
    refine_solve(A, F, b; maxiter=8, rtol=8eps)
        src/lapack/expert_refinement.jl:89-104
    inverse_norm_estimate(F; maxiter=8)
        src/lapack/expert_refinement.jl:45-60 (Hager-Higham)
    inv(A) / inv(F)
        src/api/linalg_api.jl:1143-1144 (native_inverse for a matrix,
        LinearAlgebra's inv over ldiv! for a factorization)
    factorize(A)
        src/api/linalg_api.jl:1101-1112: a dense square matrix goes to lu, a
        Hermitian one with a positive diagonal to cholesky when that succeeds;
        the other branches (QR for rectangular input, Bunch-Kaufman for other
        Hermitian input) are not part of this engine and raise ArgumentError.

Each returns what the reference returns (the NamedTuples as dicts).  All of the
arithmetic runs in liboxiblas_b200.so; there is no host fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import (ArgumentError, DimensionMismatch, Handle, SingularException, OXI_ENONFINITE,
                   OXI_ENOTCONVERGED, OXI_ESINGULAR, OXI_OK)
from .lu import LU, _as_tensor, colmajor_copy, lu

EPS = float(np.finfo(np.float64).eps)


class SolveReport(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("backward_error", ctypes.c_double),
                ("residual_norm", ctypes.c_double), ("rcond_estimate", ctypes.c_double),
                ("forward_error_estimate", ctypes.c_double), ("inverse_norm_estimate", ctypes.c_double),
                ("info", ctypes.c_int64), ("converged", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def _rhs(b, n):
    bt = _as_tensor(b)
    vec = bt.ndim == 1
    if bt.shape[0] != n:
        raise DimensionMismatch("right-hand side rows differ")
    B2 = bt.reshape(n, -1)
    return vec, B2


def _square_fp64(A):
    At = _as_tensor(A)
    if At.ndim != 2 or At.shape[0] != At.shape[1]:
        raise DimensionMismatch("matrix is not square")
    return At


def expert_solve(A, b, *, maxiter: int = 8, rtol: float = 8 * EPS, equilibrate: bool = True):
    """Equilibrated FP64 LU solve with componentwise refinement.  Returns
    dict(x, converged, iterations, backward_error, row_scale, column_scale,
    factor) where factor is the LU of the scaled matrix."""
    At = _square_fp64(A)
    n = At.shape[0]
    if maxiter < 0 or not (rtol >= 0) or not np.isfinite(rtol):
        raise ArgumentError("invalid expert solve dimensions/options")
    vec, B2 = _rhs(b, n)
    nrhs = B2.shape[1]
    Acm = colmajor_copy(At, torch.float64)
    dev = Acm.device
    rows = torch.ones(n, dtype=torch.float64, device=dev)
    cols = torch.ones(n, dtype=torch.float64, device=dev)
    Fcm = torch.empty((n, n), dtype=torch.float64, device=dev)
    ipiv = torch.zeros(max(n, 1), dtype=torch.int64, device=dev)[:n]
    Xcm = torch.zeros((nrhs, n), dtype=torch.float64, device=dev)
    Bcm = colmajor_copy(B2, torch.float64)
    h = Handle.get()
    worst = None
    it = 0
    for k0 in range(0, nrhs, 16):
        k1 = min(nrhs, k0 + 16)
        rep = SolveReport()
        st = h.lib.oxi_dexpert_solve(h.ptr, n, k1 - k0, ctypes.c_void_p(Acm.data_ptr()), max(1, n),
                                     ctypes.c_void_p(Bcm[k0:k1].data_ptr()), max(1, n),
                                     ctypes.c_void_p(Xcm[k0:k1].data_ptr()), max(1, n), int(maxiter), float(rtol),
                                     1 if equilibrate else 0, ctypes.c_void_p(rows.data_ptr()),
                                     ctypes.c_void_p(cols.data_ptr()), ctypes.c_void_p(Fcm.data_ptr()), max(1, n),
                                     ctypes.c_void_p(ipiv.data_ptr()), ctypes.byref(rep))
        if st == OXI_ESINGULAR:
            raise SingularException(rep.info)
        if st == OXI_ENONFINITE:
            raise ArgumentError("finite input required")
        if st not in (OXI_OK, OXI_ENOTCONVERGED):
            h.check(st)
        if worst is None or not (rep.backward_error <= worst):
            worst = rep.backward_error
        it = max(it, int(rep.iterations))
    X = Xcm.t()
    F = LU(Fcm, ipiv, 0, n, n)
    return dict(x=X[:, 0].clone() if vec else X.clone(), converged=bool(worst <= rtol), iterations=it,
                backward_error=float(worst), row_scale=rows, column_scale=cols, factor=F)


def _factors_of(F):
    if not isinstance(F, LU):
        raise ArgumentError("an LU factorization of this engine is required")
    if F.dtype != torch.float64:
        raise ArgumentError("FP64 factors are required")
    F._ready()
    return F


def refine_solve(A, F, b, *, maxiter: int = 8, rtol: float = 8 * EPS):
    """Iterative refinement with the factors F of A.  Returns dict(x,
    converged, iterations, backward_error, residual_norm, rcond_estimate,
    forward_error_estimate)."""
    F = _factors_of(F)
    At = _square_fp64(A)
    n = At.shape[0]
    if F.shape != (n, n):
        raise DimensionMismatch("factorization and matrix differ")
    if maxiter < 0 or not (rtol >= 0):
        raise ArgumentError("invalid refinement dimensions/options")
    vec, B2 = _rhs(b, n)
    nrhs = B2.shape[1]
    Acm = colmajor_copy(At, torch.float64)
    Bcm = colmajor_copy(B2, torch.float64)
    Xcm = torch.zeros_like(Bcm)
    rep = SolveReport()
    h = Handle.get()
    st = h.lib.oxi_drefine_solve(h.ptr, n, nrhs, ctypes.c_void_p(Acm.data_ptr()), max(1, n),
                                 ctypes.c_void_p(F._buf.data_ptr()), F._lda, ctypes.c_void_p(F.ipiv.data_ptr()),
                                 ctypes.c_void_p(Bcm.data_ptr()), max(1, n), ctypes.c_void_p(Xcm.data_ptr()),
                                 max(1, n), int(maxiter), float(rtol), ctypes.byref(rep))
    if st not in (OXI_OK, OXI_ENOTCONVERGED):
        h.check(st)
    X = Xcm.t()
    return dict(x=X[:, 0].clone() if vec else X.clone(), converged=bool(rep.converged),
                iterations=int(rep.iterations), backward_error=rep.backward_error,
                residual_norm=rep.residual_norm, rcond_estimate=rep.rcond_estimate,
                forward_error_estimate=rep.forward_error_estimate)


def inverse_norm_estimate(F, *, maxiter: int = 8) -> float:
    """Hager-Higham estimate of ||A^-1||_1 from the factors F (not a bound)."""
    F = _factors_of(F)
    if maxiter < 1:
        raise ArgumentError("invalid inverse norm estimator options")
    n = F.shape[0]
    est = ctypes.c_double(0.0)
    h = Handle.get()
    h.check(h.lib.oxi_dinverse_norm_estimate(h.ptr, n, ctypes.c_void_p(F._buf.data_ptr()), F._lda,
                                             ctypes.c_void_p(F.ipiv.data_ptr()), int(maxiter), ctypes.byref(est)))
    return est.value


def inv(A) -> torch.Tensor:
    """OxiBLAS.inv: the inverse of a square matrix (factored first) or of a
    factorization F, as an n x n CUDA tensor."""
    F = A if isinstance(A, LU) else lu(_square_fp64(A))
    if isinstance(F, LU) and F.dtype == torch.complex128:
        # ComplexF64: the solve with the identity on the complex engine
        F._ready()
        n = F.shape[0]
        return F.ldiv_(torch.eye(n, dtype=torch.complex128, device=F._buf.device))
    F = _factors_of(F)
    n = F.shape[0]
    Xcm = torch.empty((n, n), dtype=torch.float64, device=F._buf.device)
    h = Handle.get()
    h.check(h.lib.oxi_dgetri(h.ptr, n, ctypes.c_void_p(F._buf.data_ptr()), F._lda,
                             ctypes.c_void_p(F.ipiv.data_ptr()), ctypes.c_void_p(Xcm.data_ptr()), max(1, n)))
    return Xcm.t()


def _is_hermitian(At: torch.Tensor) -> bool:
    return bool(torch.equal(At, At.conj().t()))


def factorize(A):
    """OxiBLAS.factorize for a dense matrix: square and not Hermitian -> lu(A).
    Rectangular input dispatches to QR and Hermitian input to Cholesky or
    Bunch-Kaufman in the reference; neither is part of this engine."""
    if isinstance(A, LU):
        return A
    At = _as_tensor(A)
    if At.ndim != 2:
        raise DimensionMismatch("matrix expected")
    m, n = At.shape
    if m != n:
        raise ArgumentError("factorize: rectangular input dispatches to QR, which this engine does not provide")
    if _is_hermitian(At):
        # linalg_api.jl:1105-1109: a positive real diagonal tries Cholesky first
        d = torch.diagonal(At)
        if bool(torch.all(torch.isfinite(d)).item()) and bool(torch.all(d > 0).item()) and not At.is_complex():
            from .cholesky import cholesky
            C = cholesky(At, check=False)
            if C.issuccess():
                return C
        raise ArgumentError("factorize: a Hermitian matrix that is not positive definite dispatches to "
                            "Bunch-Kaufman, which this engine does not provide")
    return lu(At)
