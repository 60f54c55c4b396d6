"""Host-side mirror of OxiBLAS.jl's dense LU API over the B200 engine.

    F = lu(A; check=true)           OxiBLAS.lu             src/api/linalg_api.jl:217
    F = lu_(A; check=true)          OxiBLAS.lu!            src/api/linalg_api.jl:218
    F.L, F.U, F.p, F.P, F.factors, F.ipiv, F.info, issuccess(F)        :156-204
    ldiv_(F, B) / F.ldiv_(B)        LinearAlgebra.ldiv!(F, B)           :168-175
    F.T / F.H                       transpose(F) / F' (ldiv! on them)   :176-184
    ldiv(F, B), ldiv_into(Y, F, B)  OxiBLAS.ldiv / OxiBLAS.ldiv!   src/api/linalg_api_solve.jl:133-200
    det(F), logabsdet(F)                                               :185-191

Matrices live on the GPU as column-major buffers (a torch tensor of shape
(n, m), contiguous, is the m x n column-major matrix), exactly the layout a
Julia caller hands to the C ABI.  Indices exposed to Python are 0-based
(`p`), the LAPACK interchange sequence `ipiv` stays 1-based as in the
reference.  All arithmetic runs in liboxiblas_b200.so.
"""
from __future__ import annotations

import contextlib
import ctypes
import math

import numpy as np
import torch

from ._lib import (ArgumentError, DimensionMismatch, Handle, SingularException, OPT_BLOCKSIZE,
                   OPT_GEMM, OPT_LOOKAHEAD, OPT_TOURNAMENT, OPT_TRSM_LEAF, OXI_ESINGULAR)

_KIND = {torch.float64: "d", torch.float32: "s", torch.complex128: "z"}


def _device():
    return torch.device("cuda", torch.cuda.current_device())


def _as_tensor(A) -> torch.Tensor:
    if isinstance(A, torch.Tensor):
        t = A
    else:
        t = torch.from_numpy(np.array(A, copy=True))
    if not (t.is_floating_point() or t.is_complex()):
        t = t.to(torch.float64)  # _la_eltype: Int -> Float64 (linalg_api.jl:44)
    return t


def colmajor_copy(A, dtype=None) -> torch.Tensor:
    """Column-major device copy of a 2-D array: returns the (n, m) contiguous
    tensor whose memory is the m x n column-major matrix."""
    t = _as_tensor(A)
    if t.ndim != 2:
        raise DimensionMismatch("matrix expected")
    dev = _device()
    if t.device != dev:  # move first (a host transpose would be a slow CPU pass)
        t = t.to(dev, non_blocking=t.is_pinned())
    if dtype is not None:
        t = t.to(dtype)
    out = torch.empty((t.shape[1], t.shape[0]), dtype=t.dtype, device=dev)
    esize = {torch.float32: 4, torch.float64: 8, torch.complex128: 16}.get(t.dtype)
    if esize is not None and t.is_contiguous() and t.numel() > 0:
        # the row-major (m, n) tensor is the column-major n x m matrix t^T: the
        # engine's transpose makes the column-major m x n copy
        m, n = t.shape
        h = Handle.get()
        h.check(h.lib.oxi_transpose(h.ptr, esize, n, m, ctypes.c_void_p(t.data_ptr()), max(1, n),
                                    ctypes.c_void_p(out.data_ptr()), max(1, m)))
    else:
        out.copy_(t.t())
    return out


@contextlib.contextmanager
def options(blocksize=None, gemm=None, trsm_leaf=None, lookahead=None, tournament=None):
    """Temporarily set engine options on this thread's handle.

    blocksize  : lu_factor(...; blocksize) (reference default 128)
    gemm       : "tensor" (DMMA/tcgen05 engine, default) or "reference"
                 (one FMA chain per dot product, the reference GEMM's order)
    trsm_leaf  : leaf size of the recursive TRSM (reference 8; engine default 32)
    tournament : mixed solve only -- True: tournament pivoting in the FP32
                 factor's leaves; False (default): partial pivoting
    """
    h = Handle.get()
    saved = []
    for opt, val in ((OPT_BLOCKSIZE, blocksize), (OPT_GEMM, gemm), (OPT_TRSM_LEAF, trsm_leaf),
                     (OPT_LOOKAHEAD, lookahead), (OPT_TOURNAMENT, tournament)):
        if val is None:
            continue
        if opt == OPT_GEMM:
            val = {"tensor": 0, "reference": 1}[val] if isinstance(val, str) else int(val)
        saved.append((opt, h.get_option(opt)))
        h.set_option(opt, int(val))
    try:
        yield h
    finally:
        for opt, old in reversed(saved):
            h.set_option(opt, old)


class _AdjointLU:
    """transpose(F) / F': solves with A^T / A^H (real factors: the same solve)."""

    def __init__(self, F, trans: bytes = b"T"):
        self.parent = F
        self.trans = trans if F.dtype.is_complex else b"T"

    def ldiv_(self, B):
        return self.parent._ldiv_inplace(B, self.trans)

    def solve(self, B):
        return ldiv(self, B)

    @property
    def shape(self):
        n, m = self.parent.shape
        return (m, n)


class LU:
    """OxiBLAS.LU{T,LUFactor} on the GPU."""

    def __init__(self, buf: torch.Tensor, ipiv: torch.Tensor, info: int, m: int, n: int,
                 lda=None, factors=None):
        self._buf = buf  # (n, m) tensor whose memory is the m x n column-major matrix
        self._lda = max(1, m) if lda is None else int(lda)
        self._factors = factors  # the caller's matrix for lu_ on a column-major A
        self._ipiv = ipiv
        self._info = int(info)
        self._m, self._n = m, n
        self._perm = None

    # ---- properties (getproperty, linalg_api.jl:192-204) ----
    @property
    def shape(self):
        return (self._m, self._n)

    size = shape

    @property
    def dtype(self):
        return self._buf.dtype

    @property
    def factors(self) -> torch.Tensor:
        """m x n view holding L (strict lower, unit diagonal implicit) and U."""
        if self._factors is not None:
            return self._factors
        return self._buf.t()

    @property
    def ipiv(self) -> torch.Tensor:
        """LAPACK interchange sequence, 1-based global rows (LUFactor.pivots)."""
        return self._ipiv

    @property
    def info(self) -> int:
        return self._info

    @property
    def p(self) -> np.ndarray:
        """0-based row permutation with A[p, :] == L @ U (factorizations.jl:72-75)."""
        if self._perm is None:
            piv = self._ipiv.cpu().numpy() - 1
            p = np.arange(self._m)
            for j, pj in enumerate(piv):
                p[j], p[pj] = p[pj], p[j]
            self._perm = p
        return self._perm

    @property
    def L(self) -> torch.Tensor:
        q = min(self._m, self._n)
        f = self.factors[:, :q]
        return torch.tril(f, -1) + torch.eye(self._m, q, dtype=f.dtype, device=f.device)

    @property
    def U(self) -> torch.Tensor:
        q = min(self._m, self._n)
        return torch.triu(self.factors[:q, :])

    @property
    def P(self) -> torch.Tensor:
        """Permutation matrix with P @ A == A[p, :]."""
        m = self._m
        P = torch.zeros((m, m), dtype=self.dtype, device=self._buf.device)
        P[torch.arange(m), torch.as_tensor(self.p)] = 1
        return P

    def propertynames(self):
        return ("L", "U", "p", "P")

    def issuccess(self) -> bool:
        return self._info == 0

    @property
    def T(self):
        return _AdjointLU(self, b"T")

    @property
    def H(self):
        return _AdjointLU(self, b"C")

    def _ready(self):
        if self._m != self._n:
            raise DimensionMismatch("matrix is not square")
        if self._info != 0:
            raise SingularException(self._info)

    # ---- solves ----
    def _ldiv_inplace(self, B, trans: bytes):
        """ldiv!(F, B) / ldiv!(transpose(F), B): B overwritten and returned."""
        self._ready()
        n = self._n
        if not isinstance(B, torch.Tensor):
            raise ArgumentError("in-place solve needs a torch tensor")
        if B.shape[0] != n:
            raise DimensionMismatch(f"factorization has {n} rows, right-hand side has {B.shape[0]}")
        if B.is_complex() and not self.dtype.is_complex:
            # _apply_split!: real and imaginary parts solved separately (linalg_api.jl:67-79)
            re = B.real.to(self.dtype).clone()
            im = B.imag.to(self.dtype).clone()
            self._ldiv_inplace(re, trans)
            self._ldiv_inplace(im, trans)
            B.copy_(torch.complex(re, im))
            return B
        if B.dtype != self.dtype and self.dtype.is_complex and not B.is_complex():
            raise ArgumentError("a real right-hand side cannot hold a complex solution in place")
        if B.dtype != self.dtype or B.device != self._buf.device:
            X = B.to(device=self._buf.device, dtype=self.dtype)
            X = self._ldiv_inplace(X.clone(), trans)
            B.copy_(X)
            return B
        X2 = B.reshape(n, -1)
        nrhs = X2.shape[1]
        if nrhs == 0 or n == 0:
            return B
        cm = torch.empty((nrhs, n), dtype=self.dtype, device=self._buf.device)
        cm.copy_(X2.t())
        h = Handle.get()
        fn = {"d": h.lib.oxi_dgetrs, "s": h.lib.oxi_sgetrs, "z": h.lib.oxi_zgetrs}[_KIND[self.dtype]]
        st = fn(h.ptr, trans, n, nrhs, ctypes.c_void_p(self._buf.data_ptr()), self._lda,
                ctypes.c_void_p(self._ipiv.data_ptr()), ctypes.c_void_p(cm.data_ptr()), max(1, n))
        h.check(st)
        B.copy_(cm.t().reshape(B.shape))
        return B

    def ldiv_(self, B):
        return self._ldiv_inplace(B, b"N")

    def solve(self, B):
        return ldiv(self, B)

    # ---- determinant (linalg_api.jl:185-191) ----
    def _nswaps(self) -> int:
        piv = self._ipiv.cpu().numpy()
        return int(np.count_nonzero(piv != np.arange(1, len(piv) + 1)))

    def logabsdet(self):
        """(sum log|u_ii|, prod sign(u_ii) negated for an odd permutation);
        sign(u) = u / |u| for complex factors."""
        if self._m != self._n:
            raise DimensionMismatch("matrix is not square")
        d = torch.diagonal(self.factors)
        la = float(torch.log(torch.abs(d)).sum())
        s = torch.prod(torch.sgn(d)).item()
        if self._nswaps() % 2 == 1:
            s = -s
        return la, s

    def det(self):
        if self._m != self._n:
            raise DimensionMismatch("matrix is not square")
        d = torch.diagonal(self.factors)
        v = torch.prod(d).item()
        return -v if self._nswaps() % 2 == 1 else v


def _getrf(buf: torch.Tensor, m: int, n: int, check: bool, lda=None, factors=None) -> LU:
    """Factor the column-major matrix whose memory starts at buf.data_ptr()
    (leading dimension lda, default m)."""
    kind = _KIND.get(buf.dtype)
    if kind is None:
        raise ArgumentError(f"unsupported element type {buf.dtype}")
    lda = max(1, m) if lda is None else int(lda)
    h = Handle.get()
    q = min(m, n)
    ipiv = torch.zeros(max(q, 1), dtype=torch.int64, device=buf.device)[:q]
    info = ctypes.c_int64(0)
    fn = {"d": h.lib.oxi_dgetrf, "s": h.lib.oxi_sgetrf, "z": h.lib.oxi_zgetrf}[kind]
    st = fn(h.ptr, m, n, ctypes.c_void_p(buf.data_ptr()), lda,
            ctypes.c_void_p(ipiv.data_ptr()), ctypes.byref(info))
    if st == OXI_ESINGULAR:
        if check:
            raise SingularException(info.value)
    else:
        h.check(st)
    return LU(buf, ipiv, info.value, m, n, lda=lda, factors=factors)


def lu(A, pivot=None, *, check: bool = True, blocksize=None) -> LU:
    """OxiBLAS.lu(A, [RowMaximum()]; check=true): factors a copy of A."""
    if pivot not in (None, "RowMaximum", "rowmaximum"):
        raise ArgumentError("only partial (row-maximum) pivoting is on this path")
    buf = colmajor_copy(A)
    if buf.dtype not in _KIND:
        buf = buf.to(torch.complex128 if buf.is_complex() else torch.float64)
    m, n = buf.shape[1], buf.shape[0]
    if blocksize is not None:
        with options(blocksize=blocksize):
            return _getrf(buf, m, n, check)
    return _getrf(buf, m, n, check)


def lu_(A: torch.Tensor, *, check: bool = True, blocksize=None) -> LU:
    """OxiBLAS.lu!(A): A (a CUDA float32/float64 tensor) is overwritten by the
    factors.  For a column-major A (stride(0) == 1, any leading dimension, as a
    Julia matrix or strided view) the factorization runs in A's memory and
    F.factors is A; a row-major A is factored through a column-major copy and the
    factors are written back into A."""
    if not isinstance(A, torch.Tensor) or not A.is_cuda or A.dtype not in _KIND:
        raise TypeError("lu_ needs a CUDA float32/float64/complex128 tensor (no implicit conversion)")
    m, n = A.shape
    ctx = options(blocksize=blocksize) if blocksize is not None else contextlib.nullcontext()
    with ctx:
        if A.stride(0) == 1 and A.stride(1) >= max(1, m):
            return _getrf(A.t(), m, n, check, lda=A.stride(1), factors=A)
        buf = colmajor_copy(A)
        try:
            F = _getrf(buf, m, n, check)
        finally:
            A.copy_(buf.t())
    return F


def ldiv_(F, B):
    """LinearAlgebra.ldiv!(F, B)."""
    return F.ldiv_(B)


def ldiv(F, B):
    """OxiBLAS.ldiv(F, B): allocating solve; B is not modified."""
    parent = F.parent if isinstance(F, _AdjointLU) else F
    t = _as_tensor(B)
    if t.is_complex() and not parent.dtype.is_complex:
        Y = t.to(device=parent._buf.device).clone()
    else:
        Y = t.to(device=parent._buf.device, dtype=parent.dtype).clone()
    return F.ldiv_(Y)


def ldiv_into(Y, F, B):
    """OxiBLAS.ldiv!(Y, F, B): copy B into Y, solve in place, return Y
    (src/api/linalg_api_solve.jl:133-148)."""
    if Y is B or (isinstance(Y, torch.Tensor) and isinstance(B, torch.Tensor)
                  and Y.data_ptr() == B.data_ptr()):
        raise ArgumentError("output must not alias the right-hand side")
    Y.copy_(_as_tensor(B).to(Y.device))
    return F.ldiv_(Y)


def det(F) -> float:
    return F.det() if isinstance(F, LU) else lu(F, check=False).det()


def logabsdet(F):
    return F.logabsdet() if isinstance(F, LU) else lu(F, check=False).logabsdet()


def gemm_update(C: torch.Tensor, A: torch.Tensor, B: torch.Tensor) -> torch.Tensor:
    """gemm!(C, A, B, -1, 1): C <- C - A @ B on the FP64 tensor-core kernel.
    C, A, B: CUDA float64 tensors with unit inner stride."""
    for X in (C, A, B):
        if X.dtype != torch.float64 or not X.is_cuda or X.stride(1) != 1:
            raise ArgumentError("float64 CUDA tensors with unit inner stride required")
    m, k = A.shape
    k2, n = B.shape
    if k != k2 or C.shape != (m, n):
        raise DimensionMismatch("GEMM dimensions differ")
    h = Handle.get()
    # row-major C = (column-major C^T): C^T -= B^T A^T
    st = h.lib.oxi_dgemm_update(h.ptr, n, m, k, ctypes.c_void_p(C.data_ptr()), max(1, C.stride(0)),
                                ctypes.c_void_p(B.data_ptr()), max(1, B.stride(0)),
                                ctypes.c_void_p(A.data_ptr()), max(1, A.stride(0)))
    h.check(st)
    return C
