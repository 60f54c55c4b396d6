"""ctypes front end of the CPU parity oracle (liboxiblas_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by the tests, the smoke check and the
benchmark's CPU-baseline leg, never by the product package.  Every function
takes and returns numpy arrays in the caller's (row-index, column-index)
convention and hands the C code column-major (Fortran-ordered) copies, the
layout of the Julia reference.  Pivots are LAPACK-style 1-based global row
indices (`ipiv`), as `LUFactor.pivots` in src/lapack/factorizations.jl:5-10.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboxiblas_oracle.so")
_lib = None

_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int64)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        for P, fp in (("d", _dp), ("s", _fp)):
            f = getattr(L, f"orc_{P}getrf")
            f.argtypes = [_i64, _i64, fp, _i64, _i64, ctypes.c_int, _ip, _ip]
            f.restype = ctypes.c_int
            f = getattr(L, f"orc_{P}getrf_steps")
            f.argtypes = [_i64, _i64, fp, _i64, _i64, ctypes.c_int, _ip, _ip, _i64]
            f.restype = ctypes.c_int
            f = getattr(L, f"orc_{P}getrs")
            f.argtypes = [ctypes.c_char, _i64, _i64, fp, _i64, _ip, fp, _i64]
            f.restype = ctypes.c_int
        L.orc_refinement_residual.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64, _dp, _i64, _dp, _i64]
        L.orc_refinement_residual.restype = ctypes.c_double
        L.orc_normwise_backward_error.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64, _dp, _i64]
        L.orc_normwise_backward_error.restype = ctypes.c_double
        L.orc_equilibrate_radix.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64, _dp, _dp]
        L.orc_equilibrate_radix.restype = None
        L.orc_mixed_solve.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64, _dp, _i64, _i64,
                                      ctypes.c_double, _ip, _dp, ctypes.POINTER(ctypes.c_int)]
        L.orc_mixed_solve.restype = ctypes.c_int
        L.orc_mixed_solve_ex.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64, _dp, _i64, _i64,
                                         ctypes.c_double, ctypes.c_int, _ip, _dp, _dp,
                                         ctypes.POINTER(ctypes.c_int)]
        L.orc_mixed_solve_ex.restype = ctypes.c_int
        L.orc_inverse_norm_estimate.argtypes = [_i64, _dp, _i64, _ip, _i64]
        L.orc_inverse_norm_estimate.restype = ctypes.c_double
        L.orc_refine_solve.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64, _ip, _dp, _i64, _dp, _i64, _i64,
                                       ctypes.c_double, _dp]
        L.orc_refine_solve.restype = ctypes.c_int
        L.orc_expert_solve.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64, _dp, _i64, _i64, ctypes.c_double,
                                       ctypes.c_int, _dp, _dp, _dp, _ip, _ip, _dp]
        L.orc_expert_solve.restype = ctypes.c_int
        L.orc_inverse.argtypes = [_i64, _dp, _i64, _ip, _dp, _i64]
        L.orc_inverse.restype = ctypes.c_int
        L.orc_dpotrf.argtypes = [_i64, _dp, _i64]
        L.orc_dpotrf.restype = _i64
        L.orc_dpotrs.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64]
        L.orc_dpotrs.restype = None
        _zp = ctypes.c_void_p
        L.orc_zgetrf.argtypes = [_i64, _i64, _zp, _i64, _i64, ctypes.c_int, _ip, _ip]
        L.orc_zgetrf.restype = ctypes.c_int
        L.orc_zgetrs.argtypes = [ctypes.c_char, _i64, _i64, _zp, _i64, _ip, _zp, _i64]
        L.orc_zgetrs.restype = ctypes.c_int
        L.orc_mixed_solve_chol.argtypes = [_i64, _i64, _dp, _i64, _dp, _i64, _dp, _i64, _i64, ctypes.c_double,
                                           ctypes.c_int, _ip, _dp, _dp, ctypes.POINTER(ctypes.c_int), _ip]
        L.orc_mixed_solve_chol.restype = ctypes.c_int
        L.orc_lu_adjoint.argtypes = [_i64, _dp, _i64, _ip, _dp, _dp, _dp, _dp, _i64]
        L.orc_lu_adjoint.restype = ctypes.c_int
        for P, fp in (("d", _dp), ("s", _fp)):
            f = getattr(L, f"orc_{P}gemm_update")
            f.argtypes = [_i64, _i64, _i64, fp, _i64, fp, _i64, fp, _i64]
            f.restype = None
        L.orc_set_gemm_tiled.argtypes = [ctypes.c_int]
        L.orc_set_gemm_tiled.restype = None
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(t: int) -> None:
    lib().orc_set_num_threads(int(t))


def set_gemm_tiled(on: bool) -> None:
    """Register-tiled (default) or plain scalar trailing-update GEMM; both
    produce the same bits, element by element."""
    lib().orc_set_gemm_tiled(1 if on else 0)


class SingularError(Exception):
    """Raised where the reference throws SingularException (check=true)."""

    def __init__(self, info):
        super().__init__(f"singular: zero pivot at {info}")
        self.info = info


def getrf(A, blocksize: int = 128, check: bool = True, dtype=np.float64, steps: int = -1):
    """lu_factor(A; blocksize, check): returns (factors, ipiv, info).

    factors is an m x n array holding L (unit diagonal implicit) and U, ipiv the
    1-based global interchange sequence, info the first zero pivot (0 if none).
    """
    A = np.array(A, dtype=dtype, order="F", copy=True)
    m, n = A.shape
    q = min(m, n)
    ipiv = np.zeros(max(q, 1), dtype=np.int64)
    info = np.zeros(1, dtype=np.int64)
    P = "d" if dtype == np.float64 else "s"
    t = ctypes.c_double if dtype == np.float64 else ctypes.c_float
    f = getattr(lib(), f"orc_{P}getrf_steps")
    rc = f(m, n, _ptr(A, t), max(m, 1), blocksize, int(check), _ptr(ipiv, ctypes.c_int64),
           _ptr(info, ctypes.c_int64), steps)
    if rc == 1:
        raise SingularError(int(info[0]))
    if rc != 0:
        raise ValueError(f"oracle getrf failed ({rc})")
    return A, ipiv[:q].copy(), int(info[0])


def gemm_update(C, A, B):
    """gemm!(C, A, B, -1, 1): returns C - A @ B in the reference's order
    (one fma chain per element along k from zero, then C - s)."""
    dtype = np.asarray(C).dtype
    t = ctypes.c_double if dtype == np.float64 else ctypes.c_float
    C = np.array(C, dtype=dtype, order="F", copy=True)
    A = np.asfortranarray(A, dtype=dtype)
    B = np.asfortranarray(B, dtype=dtype)
    m, n = C.shape
    k = A.shape[1]
    f = getattr(lib(), "orc_dgemm_update" if dtype == np.float64 else "orc_sgemm_update")
    f(m, n, k, _ptr(C, t), max(m, 1), _ptr(A, t), max(m, 1), _ptr(B, t), max(k, 1))
    return C


def perm_from_ipiv(ipiv, m):
    """LUFactor.p: apply the interchanges to 1:m (src/lapack/factorizations.jl:72-75);
    returned 0-based so that A[p, :] == L @ U in numpy."""
    p = np.arange(m)
    for j, pj in enumerate(np.asarray(ipiv) - 1):
        p[j], p[pj] = p[pj], p[j]
    return p


def getrs(LU, ipiv, B, trans: str = "N"):
    """ldiv!(F, B) (trans 'N') or ldiv!(transpose(F), B) (trans 'T')."""
    LU = np.asarray(LU)
    dtype = LU.dtype
    LUf = np.array(LU, order="F", copy=False)
    vec = np.ndim(B) == 1
    X = np.array(np.reshape(B, (LU.shape[0], -1)), dtype=dtype, order="F", copy=True)
    n, nrhs = X.shape
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int64)
    P = "d" if dtype == np.float64 else "s"
    t = ctypes.c_double if dtype == np.float64 else ctypes.c_float
    rc = getattr(lib(), f"orc_{P}getrs")(trans.encode(), n, nrhs, _ptr(LUf, t), max(n, 1),
                                         _ptr(ipiv, ctypes.c_int64), _ptr(X, t), max(n, 1))
    if rc != 0:
        raise ValueError(f"oracle getrs failed ({rc})")
    return X[:, 0].copy() if vec else X


def refinement_residual(A, X, B):
    """(_refinement_residual!) -> (residual, componentwise backward error)."""
    A = np.asfortranarray(A, dtype=np.float64)
    vec = np.ndim(B) == 1
    X2 = np.asfortranarray(np.reshape(X, (A.shape[1], -1)), dtype=np.float64)
    B2 = np.asfortranarray(np.reshape(B, (A.shape[0], -1)), dtype=np.float64)
    R = np.zeros_like(B2, order="F")
    n, nrhs = B2.shape
    err = lib().orc_refinement_residual(n, nrhs, _ptr(A), max(n, 1), _ptr(X2), max(n, 1),
                                        _ptr(B2), max(n, 1), _ptr(R), max(n, 1))
    return (R[:, 0] if vec else R), err


def normwise_backward_error(A, X, B):
    A = np.asfortranarray(A, dtype=np.float64)
    X2 = np.asfortranarray(np.reshape(X, (A.shape[1], -1)), dtype=np.float64)
    B2 = np.asfortranarray(np.reshape(B, (A.shape[0], -1)), dtype=np.float64)
    n, nrhs = B2.shape
    return lib().orc_normwise_backward_error(n, nrhs, _ptr(A), max(n, 1), _ptr(X2), max(n, 1),
                                             _ptr(B2), max(n, 1))


def equilibrate_radix(A):
    """equilibrate(A; radix=true) -> (matrix, row_scale, column_scale)."""
    A = np.asfortranarray(A, dtype=np.float64)
    m, n = A.shape
    E = np.zeros_like(A, order="F")
    rows = np.ones(m)
    cols = np.ones(n)
    lib().orc_equilibrate_radix(m, n, _ptr(A), max(m, 1), _ptr(E), max(m, 1), _ptr(rows), _ptr(cols))
    return E, rows, cols


def mixed_solve(A, b, maxiter: int = 10, rtol: float = 1e-13):
    """mixed_solve(A, b; maxiter, rtol) with Float32 low factors (the reference's
    default Low).  Returns a dict with x, converged, iterations, backward_error,
    fallback."""
    A = np.asfortranarray(A, dtype=np.float64)
    n = A.shape[0]
    vec = np.ndim(b) == 1
    B = np.asfortranarray(np.reshape(b, (n, -1)), dtype=np.float64)
    nrhs = B.shape[1]
    X = np.zeros((n, nrhs), order="F")
    it = np.zeros(1, dtype=np.int64)
    err = np.zeros(1)
    fb = ctypes.c_int(0)
    rc = lib().orc_mixed_solve(n, nrhs, _ptr(A), max(n, 1), _ptr(B), max(n, 1), _ptr(X), max(n, 1),
                               maxiter, rtol, _ptr(it, ctypes.c_int64), _ptr(err), ctypes.byref(fb))
    if rc == 1:
        raise SingularError(0)
    if rc != 0:
        raise OverflowError("mixed solve conversion overflow")
    e = float(err[0])
    return dict(x=X[:, 0] if vec else X, converged=e <= rtol, iterations=int(it[0]),
                backward_error=e, fallback=bool(fb.value))


def mixed_solve_ex(A, b, maxiter: int = 10, rtol: float = 1e-13, normwise: bool = False):
    """mixed_solve with the stop test on the componentwise (reference) or the
    normwise backward error; both final errors are returned."""
    A = np.asfortranarray(A, dtype=np.float64)
    n = A.shape[0]
    vec = np.ndim(b) == 1
    B = np.asfortranarray(np.reshape(b, (n, -1)), dtype=np.float64)
    nrhs = B.shape[1]
    X = np.zeros((n, nrhs), order="F")
    it = np.zeros(1, dtype=np.int64)
    cw = np.zeros(1)
    nw = np.zeros(1)
    fb = ctypes.c_int(0)
    rc = lib().orc_mixed_solve_ex(n, nrhs, _ptr(A), max(n, 1), _ptr(B), max(n, 1), _ptr(X), max(n, 1),
                                  maxiter, rtol, 1 if normwise else 0, _ptr(it, ctypes.c_int64), _ptr(cw),
                                  _ptr(nw), ctypes.byref(fb))
    if rc == 1:
        raise SingularError(0)
    if rc != 0:
        raise OverflowError("mixed solve conversion overflow")
    e = float(nw[0] if normwise else cw[0])
    return dict(x=X[:, 0] if vec else X, converged=e <= rtol, iterations=int(it[0]),
                backward_error=float(cw[0]), backward_error_normwise=float(nw[0]), fallback=bool(fb.value))


def lu_adjoint(LU, ipiv, x, xbar):
    """(bbar, Abar) of x = A \\ b for upstream gradient xbar."""
    LU = np.asfortranarray(LU, dtype=np.float64)
    n = LU.shape[0]
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    xbar = np.ascontiguousarray(xbar, dtype=np.float64)
    bbar = np.zeros(n)
    Abar = np.zeros((n, n), order="F")
    rc = lib().orc_lu_adjoint(n, _ptr(LU), max(n, 1), _ptr(ipiv, ctypes.c_int64), _ptr(x),
                              _ptr(xbar), _ptr(bbar), _ptr(Abar), max(n, 1))
    if rc != 0:
        raise ValueError("oracle adjoint failed")
    return bbar, Abar


def inverse_norm_estimate(LU, ipiv, maxiter: int = 8) -> float:
    """inverse_norm_estimate(F, T, n; maxiter): Hager-Higham ||A^-1||_1 estimate."""
    LU = np.asfortranarray(LU, dtype=np.float64)
    n = LU.shape[0]
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int64)
    return lib().orc_inverse_norm_estimate(n, _ptr(LU), max(n, 1), _ptr(ipiv, ctypes.c_int64), maxiter)


def refine_solve(A, LU, ipiv, b, maxiter: int = 8, rtol: float = 8 * np.finfo(float).eps):
    """refine_solve(A, F, b; maxiter, rtol) -> the reference's NamedTuple as a dict."""
    A = np.asfortranarray(A, dtype=np.float64)
    LU = np.asfortranarray(LU, dtype=np.float64)
    n = A.shape[0]
    vec = np.ndim(b) == 1
    B = np.asfortranarray(np.reshape(b, (n, -1)), dtype=np.float64)
    nrhs = B.shape[1]
    X = np.zeros((n, nrhs), order="F")
    out = np.zeros(6)
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int64)
    lib().orc_refine_solve(n, nrhs, _ptr(A), max(n, 1), _ptr(LU), max(n, 1), _ptr(ipiv, ctypes.c_int64), _ptr(B),
                           max(n, 1), _ptr(X), max(n, 1), maxiter, rtol, _ptr(out))
    return dict(x=X[:, 0] if vec else X, converged=bool(out[0] <= rtol), iterations=int(out[5]),
                backward_error=float(out[0]), residual_norm=float(out[1]), rcond_estimate=float(out[2]),
                forward_error_estimate=float(out[3]), inverse_norm=float(out[4]))


def expert_solve(A, b, maxiter: int = 8, rtol: float = 8 * np.finfo(float).eps, equilibrate: bool = True):
    """expert_solve(A, b; maxiter, rtol, equilibrate) -> dict (x, converged,
    iterations, backward_error, row_scale, column_scale, factors, ipiv)."""
    A = np.asfortranarray(A, dtype=np.float64)
    n = A.shape[0]
    vec = np.ndim(b) == 1
    B = np.asfortranarray(np.reshape(b, (n, -1)), dtype=np.float64)
    nrhs = B.shape[1]
    X = np.zeros((n, nrhs), order="F")
    rows, cols = np.ones(n), np.ones(n)
    F = np.zeros((n, n), order="F")
    ipiv = np.zeros(max(n, 1), dtype=np.int64)
    info = np.zeros(1, dtype=np.int64)
    out = np.zeros(2)
    rc = lib().orc_expert_solve(n, nrhs, _ptr(A), max(n, 1), _ptr(B), max(n, 1), _ptr(X), max(n, 1), maxiter,
                                rtol, 1 if equilibrate else 0, _ptr(rows), _ptr(cols), _ptr(F),
                                _ptr(ipiv, ctypes.c_int64), _ptr(info, ctypes.c_int64), _ptr(out))
    if rc == 1:
        raise SingularError(int(info[0]))
    return dict(x=X[:, 0] if vec else X, converged=bool(out[0] <= rtol), iterations=int(out[1]),
                backward_error=float(out[0]), row_scale=rows, column_scale=cols, factors=F, ipiv=ipiv[:n].copy())


def inverse(LU, ipiv):
    """inv(F) for LU factors: the solve with the identity."""
    LU = np.asfortranarray(LU, dtype=np.float64)
    n = LU.shape[0]
    X = np.zeros((n, n), order="F")
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int64)
    lib().orc_inverse(n, _ptr(LU), max(n, 1), _ptr(ipiv, ctypes.c_int64), _ptr(X), max(n, 1))
    return X


def potrf(A):
    """cholesky_factor(A) -> (L, info): L lower (strict upper zeroed on success)."""
    L = np.array(A, dtype=np.float64, order="F", copy=True)
    n = L.shape[0]
    info = lib().orc_dpotrf(n, _ptr(L), max(n, 1))
    return L, int(info)


def potrs(L, B):
    """solve(F::CholeskyFactor, B)."""
    L = np.asfortranarray(L, dtype=np.float64)
    vec = np.ndim(B) == 1
    X = np.array(np.reshape(B, (L.shape[0], -1)), dtype=np.float64, order="F", copy=True)
    n, nrhs = X.shape
    lib().orc_dpotrs(n, nrhs, _ptr(L), max(n, 1), _ptr(X), max(n, 1))
    return X[:, 0].copy() if vec else X


def zgetrf(A, blocksize: int = 128, check: bool = False):
    """_lu_factor! for ComplexF64 -> (LU, ipiv (1-based), info)."""
    LU = np.array(A, dtype=np.complex128, order="F", copy=True)
    m, n = LU.shape
    ipiv = np.zeros(max(min(m, n), 1), dtype=np.int64)
    info = ctypes.c_int64(0)
    lib().orc_zgetrf(m, n, ctypes.c_void_p(LU.ctypes.data), max(m, 1), blocksize, 1 if check else 0,
                     _ptr(ipiv, ctypes.c_int64), ctypes.byref(info))
    return LU, ipiv[:min(m, n)], int(info.value)


def zgetrs(LU, ipiv, B, trans: str = "N"):
    """ldiv!(F, B) ('N'), ldiv!(transpose(F), B) ('T'), ldiv!(F', B) ('C')."""
    LU = np.asfortranarray(LU, dtype=np.complex128)
    vec = np.ndim(B) == 1
    X = np.array(np.reshape(B, (LU.shape[0], -1)), dtype=np.complex128, order="F", copy=True)
    n, nrhs = X.shape
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int64)
    lib().orc_zgetrs(trans.encode(), n, nrhs, ctypes.c_void_p(LU.ctypes.data), max(n, 1),
                     _ptr(ipiv, ctypes.c_int64), ctypes.c_void_p(X.ctypes.data), max(n, 1))
    return X[:, 0].copy() if vec else X


def mixed_solve_chol(A, b, maxiter: int = 10, rtol: float = 1e-13, normwise: bool = False):
    """mixed_solve(A, b; factorization=:cholesky) (Float32 Cholesky of A / max|A|,
    Float64 refinement).  Returns dict(x, converged, iterations,
    backward_error, backward_error_normwise, fallback, info)."""
    A = np.asfortranarray(A, dtype=np.float64)
    n = A.shape[0]
    vec = np.ndim(b) == 1
    B = np.asfortranarray(np.reshape(b, (n, -1)), dtype=np.float64)
    nrhs = B.shape[1]
    X = np.zeros((n, nrhs), order="F")
    it = np.zeros(1, dtype=np.int64)
    info = np.zeros(1, dtype=np.int64)
    cw = np.zeros(1)
    nw = np.zeros(1)
    fb = ctypes.c_int(0)
    rc = lib().orc_mixed_solve_chol(n, nrhs, _ptr(A), max(n, 1), _ptr(B), max(n, 1), _ptr(X), max(n, 1),
                                    maxiter, rtol, 1 if normwise else 0, _ptr(it, ctypes.c_int64), _ptr(cw),
                                    _ptr(nw), ctypes.byref(fb), _ptr(info, ctypes.c_int64))
    if rc == 1:
        raise ValueError(f"PosDefException({int(info[0])})")
    if rc != 0:
        raise OverflowError("mixed solve conversion overflow")
    e = float(nw[0] if normwise else cw[0])
    return dict(x=X[:, 0] if vec else X, converged=e <= rtol, iterations=int(it[0]),
                backward_error=float(cw[0]), backward_error_normwise=float(nw[0]), fallback=bool(fb.value),
                info=int(info[0]))
