"""GPU parity of the batched uneven LU (one persistent launch) against the oracle.

Per problem, the bars of the single-matrix tests: pivots identical to the
oracle's, factors within 1e-12 relative; solves with backward error
<= 30 * cond (test/lapack/lapack_dense.jl:15-20); the mixed mode (FP32 factor
+ FP64 refinement) reaches componentwise backward error <= 1e-13 (the
reference's mixed_solve rtol) on the batched configuration's matrices
(N(0,1) + n I, n uniform on 16..256, 1..8 right-hand sides).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


ODD_ORDERS = [1, 2, 3, 7, 8, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 200, 255, 256]


def _check_factors(P, mats, oracle, tag):
    for i, A in enumerate(mats):
        Fo, ipo, info = oracle.getrf(A, check=False)
        assert np.array_equal(_np(P.ipiv(i)), ipo), (tag, i, A.shape)
        F = _np(P.A(i))
        scale = max(1.0, np.abs(Fo).max())
        assert np.abs(F - Fo).max() <= 1e-12 * scale, (tag, i, np.abs(F - Fo).max())


@pytest.mark.parametrize("n_smem,nb", [(64, 16), (0, 8), (0, 32), (112, 16), (128, 8)])
def test_getrf_batched_matches_oracle(pkg, oracle, n_smem, nb):
    """Pivoting matrices (no diagonal shift), every panel width and both homes
    of the working matrix (shared memory up to n_smem, global beyond)."""
    rng = np.random.default_rng(31)
    mats = [rng.standard_normal((n, n)) for n in ODD_ORDERS]
    pkg.batched_set_tuning("fp64", n_smem, [nb] * 8)
    try:
        P = pkg.BatchedLU(ODD_ORDERS)
        P.load(mats)
        info = P.getrf()
        assert np.all(info == 0)
        _check_factors(P, mats, oracle, (n_smem, nb))
    finally:
        pkg.batched_set_tuning("fp64", 64, [8, 8, 16, 16, 16, 16, 16, 16])


def test_getrf_batched_singular_empty_and_invalid(pkg, oracle):
    rng = np.random.default_rng(32)
    A1 = rng.standard_normal((40, 40))
    A1[:, 5] = 0.0  # zero column: info = 6, factorization completed
    A2 = np.zeros((3, 3))
    P = pkg.BatchedLU([40, 3, 17])
    A3 = rng.standard_normal((17, 17))
    P.load([A1, A2, A3])
    info = P.getrf()
    assert list(info) == [6, 1, 0]
    Fo, ipo, info_o = oracle.getrf(A1, check=False)
    assert info_o == 6 and np.array_equal(_np(P.ipiv(0)), ipo)
    assert np.abs(_np(P.A(0)) - Fo).max() <= 1e-12 * np.abs(Fo).max()
    with pytest.raises(pkg.SingularException):
        P.load([A1, A2, A3])
        P.getrf(check=True)
    # an empty problem next to a normal one
    Q = pkg.BatchedLU([0, 5])
    Q.load([np.zeros((0, 0)), np.eye(5) * 2])
    assert list(Q.getrf()) == [0, 0]
    # order beyond 256 is refused at construction
    with pytest.raises(pkg.ArgumentError):
        pkg.BatchedLU([257])


def test_gesv_batched_fp64_solves(pkg, oracle):
    rng = np.random.default_rng(33)
    orders = ODD_ORDERS * 2
    k = rng.integers(1, 9, size=len(orders))
    mats = [rng.standard_normal((n, n)) + (0.5 * n) * np.eye(n) for n in orders]
    rhs = [rng.standard_normal((n, int(kk))) for n, kk in zip(orders, k)]
    P = pkg.BatchedLU(orders, k)
    P.load(mats, rhs)
    rep = P.gesv("fp64")
    assert np.all(rep["info"] == 0)
    for i, (A, B) in enumerate(zip(mats, rhs)):
        X = _np(P.B(i))
        ref = np.linalg.solve(A, B)
        c = np.linalg.cond(A)
        assert np.abs(X - ref).max() <= 1e-12 * c * max(1.0, np.abs(ref).max()), i
        Fo, ipo, _ = oracle.getrf(A)
        assert np.array_equal(_np(P.ipiv(i)), ipo)


def test_gesv_batched_mixed_config_subset(pkg):
    """512 problems of the batched configuration; FP32 factor + FP64 IR."""
    g = np.random.default_rng(34)
    count = 512
    orders = g.integers(16, 257, size=count)
    k = g.integers(1, 9, size=count)
    mats = [g.standard_normal((n, n)) + n * np.eye(n) for n in orders]
    rhs = [g.standard_normal((n, int(kk))) for n, kk in zip(orders, k)]
    P = pkg.BatchedLU(orders, k)
    P.load(mats, rhs)
    rep = P.gesv("fp32", maxiter=10, rtol=1e-13)
    assert rep["status"] == 0
    assert np.all(rep["info"] == 0)
    assert np.all(rep["backward_error"] <= 1e-13)
    assert rep["iterations"].max() <= 10
    for i in range(0, count, 37):
        A, B = mats[i], rhs[i]
        X = _np(P.X(i))
        R = B - A @ X
        den = np.abs(A) @ np.abs(X) + np.abs(B)
        assert (np.abs(R) / den).max() <= 1.01e-13
        assert np.allclose(_np(P.B(i)), B)  # A and B intact in mixed mode
    # same storage again: replayed as a graph, same answers
    X0 = _np(P.poolX).copy()
    rep2 = P.gesv("fp32", maxiter=10, rtol=1e-13)
    assert rep2["status"] == 0 and np.array_equal(_np(P.poolX), X0)


def test_gesv_batched_mixed_nonfinite_and_maxiter(pkg):
    rng = np.random.default_rng(35)
    A0 = rng.standard_normal((20, 20)) + 20 * np.eye(20)
    A1 = A0.copy()
    A1[3, 4] = np.inf
    P = pkg.BatchedLU([20, 20], [1, 1])
    P.load([A0, A1], [np.ones(20), np.ones(20)])
    with pytest.raises(pkg.ArgumentError):  # OXI_ENONFINITE: finite input required
        P.gesv("fp32")
    assert list(_np(P.d_info)) == [0, -2]
    P.load([A0, A0], [np.ones(20), np.ones(20)])
    rep = P.gesv("fp32", maxiter=0, rtol=0.0)
    assert rep["status"] == 8 and np.all(rep["iterations"] == 0)


def test_autotune_keeps_a_valid_tuning(pkg, oracle):
    rng = np.random.default_rng(36)
    orders = rng.integers(16, 257, size=96)
    ns, nb, ms = pkg.batched_autotune(orders, "fp64", nrhs=2)
    assert ms > 0 and 0 <= ns <= 256 and all(v in (8, 16, 32) for v in nb)
    assert pkg.batched_tuning("fp64") == (ns, nb)
    mats = [rng.standard_normal((n, n)) for n in orders[:24]]
    P = pkg.BatchedLU(orders[:24])
    P.load(mats)
    assert np.all(P.getrf() == 0)
    _check_factors(P, mats, oracle, "tuned")
    ns32, nb32, ms32 = pkg.batched_autotune(orders, "fp32", nrhs=2)
    assert ms32 > 0 and all(v in (8, 16, 32) for v in nb32)


@pytest.mark.parametrize("n_smem", [64, 0])
def test_getrf_batched_nan_pivot_rule(pkg, oracle, n_smem):
    """_lu_pivot starts from row j with strict '>' (src/lapack/factorizations.jl:
    92-107): a NaN at row j keeps row j although finite rows lie below, and a
    NaN below never wins.  Pivots must equal the oracle's (which restates it)."""
    rng = np.random.default_rng(33)
    A = rng.standard_normal((40, 40))
    A[3, 3] = np.nan          # column 3: row 3 kept
    B = rng.standard_normal((24, 24))
    B[10, 0] = np.nan         # column 0: a NaN below the diagonal never wins
    pkg.batched_set_tuning("fp64", n_smem, [16] * 8)
    try:
        P = pkg.BatchedLU([40, 24])
        P.load([A, B])
        P.getrf()
        for i, M in enumerate((A, B)):
            Fo, ipo, _ = oracle.getrf(M, check=False)
            assert np.array_equal(_np(P.ipiv(i)), ipo), i
        assert _np(P.ipiv(0))[3] == 4
    finally:
        pkg.batched_set_tuning("fp64", 64, [8, 8, 16, 16, 16, 16, 16, 16])
