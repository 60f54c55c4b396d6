"""Batched LU of many independent small matrices of uneven orders (1..256).

    P = BatchedLU(orders, nrhs)        device storage for one batch shape
    P.load(As, Bs)                     copy the matrices / right-hand sides in
    info = P.getrf()                   every A_i -> its LU factors (in place)
    X, rep = P.gesv(prec="fp64"|"fp32", maxiter=10, rtol=1e-13)
    P.adjoint(xbars)                   pullback of every X_i = A_i \\ B_i: Bbar(i), Abar(i)
    autotune(orders, prec, nrhs)       pick panel widths / shared-memory threshold

Each problem is exactly lu(A_i) / ldiv!(F_i, B_i) of the reference
(src/lapack/factorizations.jl:17-77, src/api/linalg_api.jl:168-175); the
reference has no batched LU and batches only its GEMM (gemm_batched!,
src/blas/batched.jl:4-49).  prec="fp32" is mixed_solve per problem: FP32 LU of
the radix-equilibrated matrix plus FP64 iterative refinement
(src/lapack/extended_lapack.jl:175-226).  All work is one persistent kernel
launch in liboxiblas_b200.so; a BatchedLU reused with the same storage replays
it as a CUDA graph.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import (ArgumentError, DimensionMismatch, Handle, OXI_ESINGULAR, OXI_ENOTCONVERGED,
                   SingularException)

PREC = {"fp64": 3, "fp32": 0}
NMAX, MAXRHS = 256, 8


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


class BatchedLU:
    """Device storage of a batch: each matrix column-major in one pool."""

    def __init__(self, orders, nrhs=None, device=None):
        n = np.asarray(orders, dtype=np.int64).ravel()
        if n.size == 0 or n.min() < 0 or n.max() > NMAX:
            raise ArgumentError(f"orders must lie in 0..{NMAX}")
        k = np.ones_like(n) if nrhs is None else np.asarray(nrhs, dtype=np.int64).ravel()
        if k.shape != n.shape or k.min() < 0 or k.max() > MAXRHS:
            raise ArgumentError(f"1..{MAXRHS} right-hand sides per problem")
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.count = int(n.size)
        self.orders = n
        self.nrhs = k
        self.dev = dev
        # every problem starts 16-byte aligned: sizes rounded up to 2 doubles
        offA = np.concatenate([[0], np.cumsum((n * n + 1) // 2 * 2)])
        offB = np.concatenate([[0], np.cumsum((n * k + 1) // 2 * 2)])
        self._offA, self._offB = offA, offB
        self.poolA = torch.zeros(int(offA[-1]) + 2, dtype=torch.float64, device=dev)
        self.poolB = torch.zeros(int(offB[-1]) + 2, dtype=torch.float64, device=dev)
        self.poolX = torch.zeros_like(self.poolB)
        self.poolP = torch.zeros(int(n.sum()) + 1, dtype=torch.int64, device=dev)
        offP = np.concatenate([[0], np.cumsum(n)])
        self._offP = offP
        base = lambda t: t.data_ptr()
        pa = base(self.poolA) + 8 * offA[:-1]
        pb = base(self.poolB) + 8 * offB[:-1]
        px = base(self.poolX) + 8 * offB[:-1]
        pp = base(self.poolP) + 8 * offP[:-1]
        t64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(dev)
        self.d_n = torch.from_numpy(n.astype(np.int32)).to(dev)
        self.d_nrhs = torch.from_numpy(k.astype(np.int32)).to(dev)
        self.d_ld = t64(np.maximum(n, 1))
        self.d_A, self.d_B, self.d_X, self.d_P = t64(pa), t64(pb), t64(px), t64(pp)
        self.d_info = torch.zeros(self.count, dtype=torch.int32, device=dev)
        self.d_iters = torch.zeros(self.count, dtype=torch.int32, device=dev)
        self.d_berr = torch.zeros(self.count, dtype=torch.float64, device=dev)

    # ---- views of each problem's storage (column-major n x n as (n, n).t()) ----
    def A(self, i):
        n = int(self.orders[i])
        return self.poolA[self._offA[i]:self._offA[i] + n * n].view(n, n).t()

    def B(self, i):
        n, k = int(self.orders[i]), int(self.nrhs[i])
        return self.poolB[self._offB[i]:self._offB[i] + n * k].view(k, n).t()

    def X(self, i):
        n, k = int(self.orders[i]), int(self.nrhs[i])
        return self.poolX[self._offB[i]:self._offB[i] + n * k].view(k, n).t()

    def ipiv(self, i):
        return self.poolP[self._offP[i]:self._offP[i] + int(self.orders[i])]

    def load(self, As, Bs=None):
        """Copy matrices (and right-hand sides) into the pools."""
        if len(As) != self.count:
            raise DimensionMismatch("one matrix per order expected")
        for i, a in enumerate(As):
            t = torch.as_tensor(a, dtype=torch.float64)
            if tuple(t.shape) != (int(self.orders[i]),) * 2:
                raise DimensionMismatch(f"matrix {i} has shape {tuple(t.shape)}")
            self.A(i).copy_(t)
        if Bs is not None:
            for i, b in enumerate(Bs):
                if int(self.orders[i]) == 0:
                    continue
                t = torch.as_tensor(b, dtype=torch.float64).reshape(int(self.orders[i]), -1)
                if t.shape[1] != int(self.nrhs[i]):
                    raise DimensionMismatch(f"right-hand side {i} has {t.shape[1]} columns")
                self.B(i).copy_(t)

    def getrf(self, check=False):
        """Factor every matrix in place; returns the info vector (host numpy)."""
        h = Handle.get()
        st = h.lib.oxi_dgetrf_batched_uneven(h.ptr, self.count, _vp(self.d_n), _vp(self.d_A), _vp(self.d_ld),
                                             _vp(self.d_P), _vp(self.d_info))
        info = self.d_info.cpu().numpy()
        if st == OXI_ESINGULAR:
            if check:
                raise SingularException(int(info[info > 0][0]))
        else:
            h.check(st)
        return info

    def gesv(self, prec="fp64", maxiter=10, rtol=1e-13, check=False):
        """Factor and solve every problem.  fp64: A -> factors, B -> X in place
        (X views alias B); fp32: FP32 factor + FP64 refinement, A and B intact.
        Returns a report dict with info / iterations / backward_error arrays."""
        if prec not in PREC:
            raise ArgumentError(f"prec must be one of {sorted(PREC)}")
        h = Handle.get()
        st = h.lib.oxi_dgesv_batched_uneven(h.ptr, PREC[prec], self.count, _vp(self.d_n), _vp(self.d_nrhs),
                                            _vp(self.d_A), _vp(self.d_ld), _vp(self.d_P), _vp(self.d_B),
                                            _vp(self.d_ld), _vp(self.d_X), _vp(self.d_ld), _vp(self.d_info),
                                            _vp(self.d_iters), _vp(self.d_berr), int(maxiter), float(rtol))
        rep = {"info": self.d_info.cpu().numpy(), "status": st}
        if prec == "fp32":
            rep["iterations"] = self.d_iters.cpu().numpy()
            rep["backward_error"] = self.d_berr.cpu().numpy()
        if st == OXI_ESINGULAR:
            if check:
                raise SingularException(int(rep["info"][rep["info"] > 0][0]))
        elif st != OXI_ENOTCONVERGED:
            h.check(st)
        return rep

    def solution(self, i, prec="fp64"):
        return self.B(i) if prec == "fp64" else self.X(i)

    # ---- adjoint of X_i = A_i \ B_i with the stored FP64 factors ----
    def _adjoint_pools(self):
        if not hasattr(self, "poolXbar"):
            self.poolXbar = torch.zeros_like(self.poolB)
            self.poolBbar = torch.zeros_like(self.poolB)
            self.poolAbar = torch.zeros_like(self.poolA)
            base = lambda t, off: torch.from_numpy(
                np.ascontiguousarray(t.data_ptr() + 8 * off[:-1], dtype=np.int64)).to(self.dev)
            self.d_Xbar = base(self.poolXbar, self._offB)
            self.d_Bbar = base(self.poolBbar, self._offB)
            self.d_Abar = base(self.poolAbar, self._offA)
            self.d_adj_info = torch.zeros(self.count, dtype=torch.int32, device=self.dev)

    def Xbar(self, i):
        self._adjoint_pools()
        n, k = int(self.orders[i]), int(self.nrhs[i])
        return self.poolXbar[self._offB[i]:self._offB[i] + n * k].view(k, n).t()

    def Bbar(self, i):
        self._adjoint_pools()
        n, k = int(self.orders[i]), int(self.nrhs[i])
        return self.poolBbar[self._offB[i]:self._offB[i] + n * k].view(k, n).t()

    def Abar(self, i):
        self._adjoint_pools()
        n = int(self.orders[i])
        return self.poolAbar[self._offA[i]:self._offA[i] + n * n].view(n, n).t()

    def adjoint(self, xbars=None, solution="B", check=True):
        """Pullback of every X_i = A_i \\ B_i (the rrule's bbar, Abar) with the
        FP64 factors left in the A pool by getrf() / gesv("fp64").  xbars: the
        upstream gradients (None: the Xbar pool as already filled); the
        solutions X_i are the B pool after gesv("fp64") (solution="B") or the X
        pool (solution="X").  Results: Bbar(i), Abar(i); returns the info vector."""
        self._adjoint_pools()
        if xbars is not None:
            if len(xbars) != self.count:
                raise DimensionMismatch("one upstream gradient per problem expected")
            for i, xb in enumerate(xbars):
                if int(self.orders[i]) == 0:
                    continue
                t = torch.as_tensor(xb, dtype=torch.float64).reshape(int(self.orders[i]), -1)
                self.Xbar(i).copy_(t)
        d_x = self.d_B if solution == "B" else self.d_X
        h = Handle.get()
        st = h.lib.oxi_dlu_adjoint_batched_uneven(h.ptr, self.count, _vp(self.d_n), _vp(self.d_nrhs),
                                                  _vp(self.d_A), _vp(self.d_ld), _vp(self.d_P), _vp(d_x),
                                                  _vp(self.d_ld), _vp(self.d_Xbar), _vp(self.d_ld),
                                                  _vp(self.d_Bbar), _vp(self.d_ld), _vp(self.d_Abar),
                                                  _vp(self.d_ld), _vp(self.d_adj_info))
        info = self.d_adj_info.cpu().numpy()
        if st == OXI_ESINGULAR:
            if check:
                raise SingularException(int(info[info > 0][0]))
        else:
            h.check(st)
        return info


def autotune(orders, prec="fp64", nrhs=4):
    """Tune the batched kernel on synthetic problems of these orders; returns
    (n_smem, panel widths per 32-order bucket, best ms)."""
    if prec not in PREC:
        raise ArgumentError(f"prec must be one of {sorted(PREC)}")
    h = Handle.get()
    n = np.ascontiguousarray(np.asarray(orders, dtype=np.int32).ravel())
    best = ctypes.c_double(0)
    h.check(h.lib.oxi_batched_autotune(h.ptr, PREC[prec], n.size, n.ctypes.data_as(ctypes.c_void_p), int(nrhs),
                                       ctypes.byref(best)))
    ns, nb = tuning(prec)
    return ns, nb, best.value


def tuning(prec="fp64"):
    h = Handle.get()
    ns = ctypes.c_int32(0)
    nb = (ctypes.c_int32 * 8)()
    h.check(h.lib.oxi_batched_get_tuning(h.ptr, PREC[prec], ctypes.byref(ns), nb))
    return int(ns.value), [int(v) for v in nb]


def set_tuning(prec, n_smem, nb):
    h = Handle.get()
    arr = (ctypes.c_int32 * 8)(*[int(v) for v in nb])
    h.check(h.lib.oxi_batched_set_tuning(h.ptr, PREC[prec], int(n_smem), arr))
