"""The CPU oracle against LAPACK getrf golden vectors and the reference's own
test properties (CPU only)."""
import numpy as np
import pytest

from conftest import bwd, split_lu


def test_oracle_matches_lapack_golden(oracle, golden):
    for name, c in golden.items():
        A = c["A"]
        m, n = A.shape
        F, ipiv, info = oracle.getrf(A, blocksize=c["bs"], check=False)
        assert info == c["info"], name
        # test/lapack/lapack_dense.jl:12-14: same partial-pivot choices as getrf
        if not name.startswith(("singular", "nearly_singular")):
            assert np.array_equal(ipiv, c["ipiv"]), name
        if c["lu"] is not None and info == 0:
            rel = np.linalg.norm(F - c["lu"]) / max(np.linalg.norm(c["lu"]), 1e-300)
            assert rel < 1e-13, (name, rel)
        else:
            assert abs(np.linalg.norm(F) - c["lu_fro"]) <= 1e-12 * c["lu_fro"] or info, name
        p = oracle.perm_from_ipiv(ipiv, m)
        L, U = split_lu(F, m, n)
        assert bwd(L @ U - A[p, :], A) <= 30, name


def test_oracle_singular_behaviour(oracle, golden):
    A = golden["singular_col23_40"]["A"]
    with pytest.raises(oracle.SingularError) as e:
        oracle.getrf(A)
    assert e.value.info == 23
    _, _, info = oracle.getrf(A, check=False)
    assert info == 23
    _, _, info = oracle.getrf(np.zeros((3, 3)), check=False)
    assert info == 1


def test_oracle_solves(oracle):
    rng = np.random.default_rng(5)
    for n in (1, 9, 67, 130):
        A = rng.standard_normal((n, n))
        F, ipiv, _ = oracle.getrf(A, blocksize=32)
        b = rng.standard_normal(n)
        B = rng.standard_normal((n, 3))
        x = oracle.getrs(F, ipiv, b)
        X = oracle.getrs(F, ipiv, B)
        xt = oracle.getrs(F, ipiv, b, "T")
        c = np.linalg.cond(A)
        assert bwd((A @ x - b)[:, None], A) <= 30 * c
        assert bwd(A @ X - B, A) <= 30 * c
        assert bwd((A.T @ xt - b)[:, None], A) <= 30 * c


def test_oracle_mixed_solve(oracle):
    rng = np.random.default_rng(7)
    for n in (1, 17, 67):  # test/lapack/factorizations.jl:57-63
        A = rng.standard_normal((n, n)) + n * np.eye(n)
        b = rng.standard_normal(n)
        r = oracle.mixed_solve(A, b)
        assert r["converged"] and r["iterations"] <= 10
        assert np.allclose(A @ r["x"], b, rtol=2e-12, atol=2e-12)
    r = oracle.mixed_solve(A, b, maxiter=0)  # extended_lapack tests: maxiter=0 -> not converged
    assert r["iterations"] == 0


def test_oracle_equilibrate_radix(oracle):
    rng = np.random.default_rng(11)
    A = rng.standard_normal((30, 20)) * (10.0 ** rng.uniform(-3, 3, (30, 1)))
    E, r, c = oracle.equilibrate_radix(A)
    assert np.all(np.log2(r) == np.round(np.log2(r)))
    assert np.all(np.log2(c) == np.round(np.log2(c)))
    assert np.allclose(E * r[:, None] * c[None, :], A, rtol=0, atol=0)


def test_oracle_adjoint_matches_finite_differences(oracle):
    rng = np.random.default_rng(3)
    n = 12
    A = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal(n)
    F, ipiv, _ = oracle.getrf(A)
    x = oracle.getrs(F, ipiv, b)
    bbar, Abar = oracle.lu_adjoint(F, ipiv, x, x)  # loss 0.5||x||^2 -> xbar = x
    h = 1e-6
    for _ in range(4):
        dA = rng.standard_normal((n, n))
        f = lambda M: 0.5 * np.sum(np.linalg.solve(M, b) ** 2)
        fd = (f(A + h * dA) - f(A - h * dA)) / (2 * h)
        assert abs(fd - np.sum(Abar * dA)) <= 1e-6 * max(1, abs(fd))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_tiled_gemm_is_bit_identical(oracle, dtype):
    """The register-tiled trailing update (the fast path used at benchmark
    sizes) performs, element by element, the scalar form's operations in the
    scalar form's order: factors and pivots are the same bits."""
    rng = np.random.default_rng(21)
    try:
        for (m, n, bs) in [(1000, 1000, 128), (1537, 1211, 128), (777, 1500, 64), (3000, 300, 128)]:
            A = rng.standard_normal((m, n)).astype(dtype)
            oracle.set_gemm_tiled(True)
            F1, i1, _ = oracle.getrf(A, blocksize=bs, dtype=dtype, check=False)
            oracle.set_gemm_tiled(False)
            F2, i2, _ = oracle.getrf(A, blocksize=bs, dtype=dtype, check=False)
            assert np.array_equal(i1, i2) and np.array_equal(F1, F2), (m, n, bs)
            C = rng.standard_normal((301, 203)).astype(dtype)
            Am = rng.standard_normal((301, 77)).astype(dtype)
            Bm = rng.standard_normal((77, 203)).astype(dtype)
            oracle.set_gemm_tiled(True)
            G1 = oracle.gemm_update(C, Am, Bm)
            oracle.set_gemm_tiled(False)
            G2 = oracle.gemm_update(C, Am, Bm)
            assert np.array_equal(G1, G2)
    finally:
        oracle.set_gemm_tiled(True)


def test_oracle_expert_solves(oracle):
    """The oracle's expert_solve / refine_solve / inverse_norm_estimate against
    the reference's properties (test/lapack/expert_* style checks)."""
    rng = np.random.default_rng(17)
    n = 120
    A = rng.standard_normal((n, n)) * (10.0 ** rng.uniform(-3, 3, (n, 1)))
    b = rng.standard_normal(n)
    r = oracle.expert_solve(A, b)
    assert r["converged"] and r["backward_error"] <= 8 * np.finfo(float).eps
    assert np.all(r["row_scale"] > 0) and np.all(r["column_scale"] > 0)
    F, ip, _ = oracle.getrf(A)
    est = oracle.inverse_norm_estimate(F, ip)
    true = np.linalg.norm(np.linalg.inv(A), 1)
    assert true / 3 <= est <= true * (1 + 1e-10)
    rs = oracle.refine_solve(A, F, ip, b)
    assert rs["converged"]
    assert np.isclose(rs["rcond_estimate"], 1 / (np.linalg.norm(A, 1) * est), rtol=1e-12)
    X = oracle.inverse(F, ip)
    assert np.allclose(X @ A, np.eye(n), atol=1e-8)


def _py_zgetf2(A):
    """Unblocked complex LU by the pivot rule of _lu_pivot (abs2 with strict
    '>', abs when the largest square is not finite; factorizations.jl:92-107)
    in plain Python loops, an independent restatement for small cases."""
    with np.errstate(over="ignore", invalid="ignore"):
        return _py_zgetf2_body(np.array(A, dtype=np.complex128))


def _py_zgetf2_body(A):
    m, n = A.shape
    piv = []
    for j in range(min(m, n)):
        p, best = j, A[j, j].real ** 2 + A[j, j].imag ** 2
        for i in range(j + 1, m):
            v = A[i, j].real ** 2 + A[i, j].imag ** 2
            if v > best:
                best, p = v, i
        if not np.isfinite(best):
            p, best = j, abs(A[j, j])
            for i in range(j + 1, m):
                v = abs(A[i, j])
                if v > best:
                    best, p = v, i
        piv.append(p + 1)
        A[[j, p], :] = A[[p, j], :]
        d = A[j, j]
        if d == 0:
            continue
        A[j + 1:, j] /= d
        A[j + 1:, j + 1:] -= np.outer(A[j + 1:, j], A[j, j + 1:])
    return A, np.array(piv, dtype=np.int64)


@pytest.mark.parametrize("m,n", [(12, 12), (40, 25), (25, 40), (70, 70)])
def test_oracle_complex_lu(oracle, m, n):
    rng = np.random.default_rng(m * n)
    A = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    LU, ipiv, info = oracle.zgetrf(A, blocksize=16)
    F2, piv2 = _py_zgetf2(A)
    assert info == 0
    assert np.array_equal(ipiv, piv2)
    assert np.linalg.norm(LU - F2) <= 1e-13 * np.linalg.norm(F2)
    q = min(m, n)
    L = np.tril(LU[:, :q], -1) + np.eye(m, q)
    U = np.triu(LU[:q, :])
    p = oracle.perm_from_ipiv(ipiv, m)
    assert bwd(L @ U - A[p, :], A) <= 30
    assert np.all(np.abs(L) <= 1 + 1e-12)  # the largest-modulus pivot
    if m == n:
        b = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
        for t, M in (("N", A), ("T", A.T), ("C", A.conj().T)):
            x = oracle.zgetrs(LU, ipiv, b, t)
            assert np.linalg.norm(M @ x - b) <= 1e-10 * np.linalg.norm(M) * np.linalg.norm(x)


def test_oracle_complex_pivot_overflow_and_zero(oracle):
    rng = np.random.default_rng(11)
    A = rng.standard_normal((20, 20)) + 1j * rng.standard_normal((20, 20))
    A[3, 0] = 3e200 + 1e200j
    A[9, 0] = 1e200 - 3.1e200j  # larger modulus; both squares overflow
    _, ipiv, _ = oracle.zgetrf(A)
    _, piv2 = _py_zgetf2(A)
    assert ipiv[0] == 10 and np.array_equal(ipiv, piv2)
    S = A.copy()
    S[:, 4] = 0
    S[3, 0], S[9, 0] = 1.0, 2.0
    _, _, info = oracle.zgetrf(S, check=False)
    assert info == 5


def test_oracle_mixed_cholesky(oracle):
    rng = np.random.default_rng(21)
    n = 200
    G = rng.standard_normal((n, n))
    A = G @ G.T + n * np.eye(n)
    b = rng.standard_normal(n)
    r = oracle.mixed_solve_chol(A, b, maxiter=20, rtol=1e-13)
    assert r["converged"] and not r["fallback"]
    x = np.linalg.solve(A, b)
    assert np.linalg.norm(r["x"] - x) <= 1e-11 * np.linalg.norm(x)
    N = A.copy()
    N[50, 50] = -1.0
    with pytest.raises(ValueError):
        oracle.mixed_solve_chol(N, b)
