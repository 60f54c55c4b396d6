"""Bounded device waits: one wait that runs out ends the whole call quickly.

The failure is made on the host, in the allowed form: a one-shot test hook
(OXI_OPT_TEST_MISSING_PRODUCER) launches, before the k-th leaf of the next
factorization, a consumer that waits for a flag no kernel ever sets.  With a
short wait limit (OXI_OPT_WAIT_LIMIT_US) that wait gives up, sets the call's
sticky abort word, and every later leaf, GEMM and triangular solve of the call
returns at its entry.  The call must come back with OXI_ETIMEOUT after about
one wait limit (not one per launch), and the handle and context must stay
usable: the next call on the same handle factors correctly.
"""
import ctypes
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LIMIT_US = 50_000  # 50 ms


def _fresh_handle(pkg):
    from oxiblas_b200 import _lib
    h = _lib.Handle()
    h.lib.oxi_set_stream(h.ptr, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return h


def _colmajor(A):
    return torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # storage = A column-major


def _getrf(h, dA, n):
    ipiv = torch.zeros(n, dtype=torch.int64, device="cuda")
    info = ctypes.c_int64(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = h.lib.oxi_dgetrf(h.ptr, n, n, ctypes.c_void_p(dA.data_ptr()), n, ctypes.c_void_p(ipiv.data_ptr()),
                          ctypes.byref(info))
    dt = time.perf_counter() - t0
    return st, dt, ipiv


@pytest.mark.parametrize("stall_leaf", [1, 7])
def test_missing_producer_ends_factorization_fast(pkg, oracle, stall_leaf):
    from oxiblas_b200 import _lib
    n = 2048  # 16 panels x 4 leaves of the FP64 path
    rng = np.random.default_rng(5)
    A = rng.standard_normal((n, n))
    h = _fresh_handle(pkg)
    try:
        h.set_option(_lib.OPT_WAIT_LIMIT_US, LIMIT_US)
        assert h.get_option(_lib.OPT_WAIT_LIMIT_US) == LIMIT_US
        st, dt0, _ = _getrf(h, _colmajor(A), n)  # warm: kernels loaded, workspace sized
        assert st == _lib.OXI_OK
        h.set_option(_lib.OPT_TEST_MISSING_PRODUCER, stall_leaf)
        st, dt, _ = _getrf(h, _colmajor(A), n)
        assert st == _lib.OXI_ETIMEOUT, st
        assert b"missing producer" in h.lib.oxi_last_error(h.ptr)
        # one wait limit, plus the launches that return at entry: far below the
        # 2 s per remaining leaf that a non-sticky timeout would cost
        assert dt < 1.0, dt
        assert h.get_option(_lib.OPT_TEST_MISSING_PRODUCER) == 0  # one-shot
        # the context and the handle are still usable
        st, _, ipiv = _getrf(h, _colmajor(A), n)
        assert st == _lib.OXI_OK
        _, ipo, _ = oracle.getrf(A)
        assert np.array_equal(ipiv.cpu().numpy(), ipo)
    finally:
        h.lib.oxi_destroy(h.ptr)


def test_missing_producer_ends_mixed_solve_fast(pkg):
    """The mixed solve's FP32 factor (tensor-core trailing updates on a second
    stream) also stops at the first expired wait and reports OXI_ETIMEOUT."""
    from oxiblas_b200 import _lib
    n = 4096
    rng = np.random.default_rng(6)
    A = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal(n)
    h = _fresh_handle(pkg)
    try:
        h.set_option(_lib.OPT_WAIT_LIMIT_US, LIMIT_US)
        dA = _colmajor(A)
        dB = torch.from_numpy(b).cuda()
        dX = torch.zeros(n, dtype=torch.float64, device="cuda")
        rep = ctypes.create_string_buffer(256)

        def solve():
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = h.lib.oxi_dgesv_mixed(h.ptr, 5, 2, n, 1, ctypes.c_void_p(dA.data_ptr()), n,
                                       ctypes.c_void_p(dB.data_ptr()), n, ctypes.c_void_p(dX.data_ptr()), n,
                                       10, 1e-13, rep)
            return st, time.perf_counter() - t0

        assert solve()[0] == _lib.OXI_OK
        h.set_option(_lib.OPT_TEST_MISSING_PRODUCER, 20)
        st, dt = solve()
        assert st == _lib.OXI_ETIMEOUT, st
        assert dt < 1.0, dt
        st, _ = solve()
        assert st == _lib.OXI_OK
        x = dX.cpu().numpy()
        assert np.linalg.norm(A @ x - b) / (np.linalg.norm(A) * np.linalg.norm(x)) < 1e-14
    finally:
        h.lib.oxi_destroy(h.ptr)


def test_wait_limit_option_bounds(pkg):
    from oxiblas_b200 import _lib
    h = _fresh_handle(pkg)
    try:
        assert h.get_option(_lib.OPT_WAIT_LIMIT_US) == 2_000_000  # default 2 s
        with pytest.raises(_lib.ArgumentError):
            h.set_option(_lib.OPT_WAIT_LIMIT_US, 10)  # below 1 ms
        with pytest.raises(_lib.ArgumentError):
            h.set_option(_lib.OPT_TEST_MISSING_PRODUCER, -1)
    finally:
        h.lib.oxi_destroy(h.ptr)
