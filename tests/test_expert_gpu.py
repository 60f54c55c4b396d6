"""expert_solve, refine_solve, inverse_norm_estimate, inv and factorize on the
GPU against the oracle's restatements of the reference
(src/lapack/advanced_factorizations.jl:591-645, src/lapack/expert_refinement.jl:
45-60 and 89-104, src/api/linalg_api.jl:1101-1112 and 1143-1144) and against
the reference's own properties."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
EPS = np.finfo(float).eps


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("n,nrhs", [(200, 1), (1000, 3), (2048, 16)])
def test_expert_solve_matches_oracle(pkg, oracle, n, nrhs):
    rng = np.random.default_rng(n + nrhs)
    A = rng.standard_normal((n, n)) * (10.0 ** rng.uniform(-4, 4, (n, 1)))  # badly row-scaled
    b = rng.standard_normal((n, nrhs)) if nrhs > 1 else rng.standard_normal(n)
    r = pkg.expert_solve(A, b)
    o = oracle.expert_solve(A, b)
    # the scales and the factorization of the scaled matrix: the same bits
    assert np.array_equal(_np(r["row_scale"]), o["row_scale"])
    assert np.array_equal(_np(r["column_scale"]), o["column_scale"])
    assert np.array_equal(_np(r["factor"].ipiv), o["ipiv"])
    assert np.array_equal(_np(r["factor"].factors), o["factors"])
    assert r["converged"] and r["backward_error"] <= 8 * EPS
    assert r["iterations"] <= 8
    x = _np(r["x"])
    _, berr = oracle.refinement_residual(A, x, b)
    assert berr <= 8 * EPS
    xo = o["x"]
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-12


def test_expert_solve_zero_row_and_no_equilibration(pkg, oracle):
    rng = np.random.default_rng(3)
    A = rng.standard_normal((50, 50))
    A[17, :] = 0.0
    with pytest.raises(pkg.SingularException) as e:
        pkg.expert_solve(A, rng.standard_normal(50))
    assert e.value.info == 18
    with pytest.raises(oracle.SingularError):
        oracle.expert_solve(A, rng.standard_normal(50))
    B = rng.standard_normal((120, 120)) + 120 * np.eye(120)
    b = rng.standard_normal(120)
    r = pkg.expert_solve(B, b, equilibrate=False)
    o = oracle.expert_solve(B, b, equilibrate=False)
    assert np.all(_np(r["row_scale"]) == 1) and np.all(_np(r["column_scale"]) == 1)
    assert np.array_equal(_np(r["factor"].factors), o["factors"])
    assert r["converged"]
    r0 = pkg.expert_solve(B, b, maxiter=0, rtol=0.0)
    assert not r0["converged"] and r0["iterations"] == 0


@pytest.mark.parametrize("n", [300, 1500])
def test_refine_solve_and_condition_estimate(pkg, oracle, n):
    rng = np.random.default_rng(n)
    A = np.asarray(_np(pkg.synthetic.kappa_matrix(n, 1e6, seed=n)))
    b = rng.standard_normal(n)
    F = pkg.lu(A)
    r = pkg.refine_solve(A, F, b)
    Fo, ipo, _ = oracle.getrf(A)
    o = oracle.refine_solve(A, Fo, ipo, b)
    assert r["converged"] and r["backward_error"] <= 8 * EPS, r
    assert abs(r["rcond_estimate"] - o["rcond_estimate"]) <= 1e-10 * o["rcond_estimate"]
    true_rcond = 1.0 / (np.linalg.norm(A, 1) * np.linalg.norm(np.linalg.inv(A), 1))
    assert true_rcond * (1 - 1e-8) <= r["rcond_estimate"] <= 3.0 * true_rcond
    assert 0 <= r["forward_error_estimate"] < 1e-6
    assert r["residual_norm"] >= 0
    # the estimator alone, against the oracle and the true norm
    est = pkg.inverse_norm_estimate(F)
    esto = oracle.inverse_norm_estimate(Fo, ipo)
    true = np.linalg.norm(np.linalg.inv(A), 1)
    assert abs(est - esto) <= 1e-10 * esto
    assert true / 3 <= est <= true * (1 + 1e-10)


def test_inv_and_factorize(pkg, oracle):
    rng = np.random.default_rng(9)
    n = 700
    A = rng.standard_normal((n, n))
    Xi = _np(pkg.inv(A))
    F = pkg.lu(A)
    Xi2 = _np(pkg.inv(F))
    assert np.array_equal(Xi, Xi2)
    ref = np.linalg.inv(A)
    c = np.linalg.cond(A, 1)
    assert np.linalg.norm(Xi - ref, 1) / np.linalg.norm(ref, 1) <= 100 * c * EPS
    Fo, ipo, _ = oracle.getrf(A)
    Xo = oracle.inverse(Fo, ipo)
    assert np.linalg.norm(Xi - Xo, 1) / np.linalg.norm(Xo, 1) <= 100 * c * EPS
    G = pkg.factorize(A)
    assert isinstance(G, pkg.LU) and np.array_equal(_np(G.factors), Fo)
    with pytest.raises(pkg.ArgumentError):
        pkg.factorize(rng.standard_normal((5, 4)))
    S = rng.standard_normal((6, 6))
    with pytest.raises(pkg.ArgumentError):
        pkg.factorize(S + S.T - 20 * np.eye(6))  # Hermitian, negative diagonal: Bunch-Kaufman
    C = pkg.factorize(S @ S.T + 6 * np.eye(6))  # Hermitian positive definite: Cholesky
    assert isinstance(C, pkg.Cholesky) and C.issuccess()
    with pytest.raises(pkg.SingularException):
        pkg.inv(np.zeros((4, 4)))
