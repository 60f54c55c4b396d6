"""oxi_dgetrs_noalloc against oxi_dgetrs, both called through the C ABI.

The no-allocation entry point keeps its scratch in one file-scope device array
that every call shares; two calls in a row (a larger system, then a smaller
one with the other transpose) must each give what oxi_dgetrs gives, within the
1e-12 relative bar of the factor parity tests.  The file name sorts last so the
test runs after the others in a full run; it also passes alone in a fresh
process (its first call does the per-device set-up).
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

OXI_ESCRATCH = 9
NOALLOC_MAX_ELEMS = 917504


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _factor(pkg, h, A):
    """Column-major device copy of A factored by oxi_dgetrf."""
    n = A.shape[0]
    LU = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # memory = A column-major
    ipiv = torch.empty(n, dtype=torch.int64, device="cuda")
    info = ctypes.c_int64(0)
    h.check(h.lib.oxi_dgetrf(h.ptr, n, n, _vp(LU), n, _vp(ipiv), ctypes.byref(info)))
    assert info.value == 0
    return LU, ipiv


def test_noalloc_getrs_matches_getrs_twice(pkg):
    h = pkg.Handle.get()
    L = h.lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(11)
    cases = []
    for n, nrhs, trans in ((777, 3, b"N"), (300, 1, b"T")):
        A = rng.standard_normal((n, n)) + 2 * np.eye(n)
        B = rng.standard_normal((nrhs, n))  # rows of this array = columns of B (column-major)
        LU, ipiv = _factor(pkg, h, A)
        Bref = torch.from_numpy(B).cuda()
        h.check(L.oxi_dgetrs(h.ptr, trans, n, nrhs, _vp(LU), n, _vp(ipiv), _vp(Bref), n))
        cases.append((n, nrhs, trans, A, B, LU, ipiv, Bref.cpu().numpy()))
    for n, nrhs, trans, A, B, LU, ipiv, Xref in cases:  # two no-allocation calls in a row
        Bna = torch.from_numpy(B).cuda()
        st = L.oxi_dgetrs_noalloc(stream, trans, n, nrhs, _vp(LU), n, _vp(ipiv), _vp(Bna), n)
        assert st == 0, L.oxi_status_string(st)
        X = Bna.cpu().numpy()
        scale = max(1.0, np.abs(Xref).max())
        assert np.abs(X - Xref).max() <= 1e-12 * scale, (n, trans, np.abs(X - Xref).max())
        M = A if trans == b"N" else A.T
        assert np.allclose(M @ X.T, B.T, rtol=1e-9, atol=1e-9)


def test_noalloc_rejects_sizes_beyond_its_scratch(pkg):
    h = pkg.Handle.get()
    L = h.lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 512
    nrhs = NOALLOC_MAX_ELEMS // n + 1
    rng = np.random.default_rng(12)
    LU, ipiv = _factor(pkg, h, rng.standard_normal((n, n)) + 2 * np.eye(n))
    B = torch.ones((nrhs, n), dtype=torch.float64, device="cuda")
    st = L.oxi_dgetrs_noalloc(stream, b"N", n, nrhs, _vp(LU), n, _vp(ipiv), _vp(B), n)
    assert st == OXI_ESCRATCH
    assert b"scratch" in L.oxi_status_string(st)
    assert bool((B == 1).all())  # nothing launched


def test_noalloc_many_rhs_matches_getrs(pkg):
    """nrhs = 19: several launches of the solve kernels (8 + 8 + 2 + 1
    columns) reuse the one scratch array within a call."""
    h = pkg.Handle.get()
    L = h.lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(13)
    n, nrhs = 1500, 19
    A = rng.standard_normal((n, n)) + 2 * np.eye(n)
    B = rng.standard_normal((nrhs, n))
    LU, ipiv = _factor(pkg, h, A)
    for trans in (b"N", b"T"):
        Bref = torch.from_numpy(B).cuda()
        h.check(L.oxi_dgetrs(h.ptr, trans, n, nrhs, _vp(LU), n, _vp(ipiv), _vp(Bref), n))
        Bna = torch.from_numpy(B).cuda()
        assert L.oxi_dgetrs_noalloc(stream, trans, n, nrhs, _vp(LU), n, _vp(ipiv), _vp(Bna), n) == 0
        Xref = Bref.cpu().numpy()
        assert np.abs(Bna.cpu().numpy() - Xref).max() <= 1e-12 * max(1.0, np.abs(Xref).max())


def test_noalloc_largest_order_on_a_permutation_factor(pkg):
    """n = OXI_NOALLOC_MAX_N (65536), one right-hand side, on a cheap factor:
    L = U = I with a random interchange sequence, so X is the permuted B.  This
    exercises the shared-memory permutation kernel at its 16-bit-row limit."""
    h = pkg.Handle.get()
    L = h.lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 65536
    rng = np.random.default_rng(14)
    LU = torch.eye(n, dtype=torch.float64, device="cuda")  # 34 GB: symmetric, so its memory is column-major I
    ipiv_h = np.array([rng.integers(j + 1, n + 1) for j in range(n)], dtype=np.int64)
    ipiv = torch.from_numpy(ipiv_h).cuda()
    b = rng.standard_normal(n)
    p = np.arange(n)
    for j, pj in enumerate(ipiv_h - 1):
        p[j], p[pj] = p[pj], p[j]
    B = torch.from_numpy(b.copy()).cuda()
    assert L.oxi_dgetrs_noalloc(stream, b"N", n, 1, _vp(LU), n, _vp(ipiv), _vp(B), n) == 0
    assert np.array_equal(B.cpu().numpy(), b[p])  # L U x = P b with L = U = I
    Bref = torch.from_numpy(b.copy()).cuda()
    h.check(L.oxi_dgetrs(h.ptr, b"N", n, 1, _vp(LU), n, _vp(ipiv), _vp(Bref), n))
    assert torch.equal(B, Bref)
    del LU
    torch.cuda.empty_cache()


def test_noalloc_invalid_pivot_leaves_b_untouched(pkg):
    h = pkg.Handle.get()
    L = h.lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(15)
    n = 200
    LU, ipiv = _factor(pkg, h, rng.standard_normal((n, n)) + 2 * np.eye(n))
    bad = ipiv.clone()
    bad[57] = n + 3  # out of range
    B = torch.from_numpy(rng.standard_normal((2, n))).cuda()
    B0 = B.clone()
    st = L.oxi_dgetrs_noalloc(stream, b"N", n, 2, _vp(LU), n, _vp(bad), _vp(B), n)
    assert st == 1  # OXI_EINVAL
    assert torch.equal(B, B0)


def test_noalloc_call_allocates_no_device_memory(pkg):
    """After a first (set-up) call, a call leaves the device's free memory
    exactly as it was: no cudaMalloc, no allocating library routine."""
    h = pkg.Handle.get()
    L = h.lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(16)
    n, nrhs = 900, 5
    LU, ipiv = _factor(pkg, h, rng.standard_normal((n, n)) + 2 * np.eye(n))
    B = torch.from_numpy(rng.standard_normal((nrhs, n))).cuda()
    assert L.oxi_dgetrs_noalloc(stream, b"N", n, nrhs, _vp(LU), n, _vp(ipiv), _vp(B), n) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for trans in (b"N", b"T", b"N"):
        assert L.oxi_dgetrs_noalloc(stream, trans, n, nrhs, _vp(LU), n, _vp(ipiv), _vp(B), n) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
