"""OxiBLAS.cholesky / cholesky! on the B200 engine (FP64).

    F = cholesky(A; check=True)       A Hermitian (real symmetric) positive definite
    F = cholesky_(A)                  in place: A's lower triangle becomes L
    F.L, F.U, F.UL, F.uplo, F.factors, F.info, issuccess(F)
    x = F.solve(b) / F.ldiv_(B)       ldiv!(F, B): L y = b, L^T x = y
    logabsdet(F), det(F)

Mirrors src/api/linalg_api.jl:221-290 (the Cholesky{T,E} wrapper of
cholesky_factor, src/lapack/factorizations.jl:205-305): a matrix that is not
symmetric raises PosDefException(-1), a pivot that is not finite and positive
PosDefException(j) (check=True) or gives issuccess(F) == False (check=False).
The factorization and the solves run in liboxiblas_b200.so (oxi_dpotrf /
oxi_dpotrs).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import ArgumentError, DimensionMismatch, Handle
from .lu import _as_tensor, colmajor_copy

OXI_ENOTPOSDEF = 10


class PosDefException(Exception):
    """LinearAlgebra.PosDefException(info): the leading minor of order info is
    not positive definite (-1: the input is not Hermitian)."""

    def __init__(self, info: int):
        super().__init__(f"PosDefException({info})")
        self.info = int(info)


class Cholesky:
    """OxiBLAS.Cholesky{T,CholeskyFactor} on the GPU (lower factor)."""

    def __init__(self, buf: torch.Tensor, n: int, info: int, lda=None):
        self._buf = buf  # (n, lda) tensor whose memory is the n x n column-major factor
        self._lda = max(1, n) if lda is None else int(lda)
        self._n = n
        self._info = int(info)

    @property
    def shape(self):
        return (self._n, self._n)

    size = shape

    @property
    def factors(self) -> torch.Tensor:
        return self._buf[:, :self._n].t() if self._buf.shape[1] != self._n else self._buf.t()

    @property
    def L(self) -> torch.Tensor:
        return torch.tril(self.factors)

    UL = L

    @property
    def U(self) -> torch.Tensor:
        return self.L.t()

    @property
    def uplo(self) -> str:
        return "L"

    @property
    def info(self) -> int:
        return self._info

    def propertynames(self):
        return ("L", "U", "UL")

    def issuccess(self) -> bool:
        return self._info == 0

    def _ready(self):
        if self._info != 0:
            raise PosDefException(self._info)

    def ldiv_(self, B: torch.Tensor) -> torch.Tensor:
        """ldiv!(F, B): B (a float64 CUDA tensor, n or n x k) overwritten by A^-1 B."""
        self._ready()
        n = self._n
        if not isinstance(B, torch.Tensor):
            raise ArgumentError("in-place solve needs a torch tensor")
        if B.shape[0] != n:
            raise DimensionMismatch(f"factorization has {n} rows, right-hand side has {B.shape[0]}")
        X2 = B.reshape(n, -1)
        nrhs = X2.shape[1]
        if n == 0 or nrhs == 0:
            return B
        cm = torch.empty((nrhs, n), dtype=torch.float64, device=self._buf.device)
        cm.copy_(X2.t())
        h = Handle.get()
        h.check(h.lib.oxi_dpotrs(h.ptr, n, nrhs, ctypes.c_void_p(self._buf.data_ptr()), self._lda,
                                 ctypes.c_void_p(cm.data_ptr()), max(1, n)))
        B.copy_(cm.t().reshape(B.shape))
        return B

    def solve(self, B):
        Bt = _as_tensor(B).to(device=self._buf.device, dtype=torch.float64).clone()
        return self.ldiv_(Bt)

    def logabsdet(self):
        """(log|det A|, sign) = (2 sum log L_ii, 1) (linalg_api.jl:248-252)."""
        self._ready()
        d = torch.diagonal(self.factors)
        return 2.0 * float(torch.log(d).sum()), 1.0

    def det(self) -> float:
        la, s = self.logabsdet()
        return s * float(np.exp(la))


def _potrf(buf: torch.Tensor, n: int, check: bool, lda=None) -> Cholesky:
    h = Handle.get()
    info = ctypes.c_int64(0)
    lda = max(1, n) if lda is None else int(lda)
    st = h.lib.oxi_dpotrf(h.ptr, n, ctypes.c_void_p(buf.data_ptr()), lda, ctypes.byref(info))
    if st == OXI_ENOTPOSDEF:
        if check:
            raise PosDefException(info.value)
    else:
        h.check(st)
    return Cholesky(buf, n, info.value, lda)


def cholesky(A, pivot=None, *, check: bool = True) -> Cholesky:
    """OxiBLAS.cholesky(A, [NoPivot()]; check=true): factors a copy of A's
    lower triangle.  A must be symmetric (Hermitian); otherwise
    PosDefException(-1) (check) or a failed factorization with info -1."""
    if pivot not in (None, "NoPivot", "nopivot"):
        raise ArgumentError("only the unpivoted Cholesky factorization is on this path")
    At = _as_tensor(A)
    if At.ndim != 2 or At.shape[0] != At.shape[1]:
        raise DimensionMismatch("matrix is not square")
    if At.is_complex():
        raise ArgumentError("complex Cholesky is not part of this engine")
    buf = colmajor_copy(At, torch.float64)
    n = At.shape[0]
    if not bool(torch.equal(buf, buf.t())):  # LinearAlgebra.ishermitian
        if check:
            raise PosDefException(-1)
        return Cholesky(buf, n, -1)
    return _potrf(buf, n, check)


def cholesky_(A: torch.Tensor, *, check: bool = True) -> Cholesky:
    """OxiBLAS.cholesky!(A): A (a float64 CUDA tensor whose memory is the
    column-major matrix, e.g. M.t() of a row-major M) has its lower triangle
    overwritten by L and its strict upper triangle zeroed.  Only the lower
    triangle is read."""
    if not isinstance(A, torch.Tensor) or not A.is_cuda or A.dtype != torch.float64:
        raise ArgumentError("cholesky_ needs a float64 CUDA tensor")
    n = A.shape[0]
    if A.ndim != 2 or A.shape[1] != n:
        raise DimensionMismatch("matrix is not square")
    if A.stride(0) != 1:
        raise ArgumentError("cholesky_ needs column-major storage (A.stride(0) == 1)")
    F = _potrf(A.t(), n, check, lda=A.stride(1))
    return F
