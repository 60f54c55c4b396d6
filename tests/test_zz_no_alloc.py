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
