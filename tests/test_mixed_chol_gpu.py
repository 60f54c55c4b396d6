"""mixed_solve(A, b; factorization=:cholesky) on the GPU (oxi_dposv_mixed)
against the oracle's restatement of _mixed_precision_impl's Cholesky family
(src/lapack/extended_lapack.jl:175-226: one global scale max|a_ij|, the Float32
Cholesky of A / scale, Float64 refinement with the corrections of
_mixed_extended_correction, fallback to the Float64 factor).

Bars: converged to rtol; the componentwise backward error (checked on the host
in FP64) <= rtol; with the FP32 factor the iteration count within one of the
oracle's and the answer within a conditioned tolerance of the oracle's; the
fallback and PosDefException cases as the reference takes them.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _spd(rng, n, cond=None):
    if cond is None:
        G = rng.standard_normal((n, n))
        return G @ G.T + n * np.eye(n)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = 10.0 ** (-np.log10(cond) * rng.uniform(0, 1, n))
    s[0], s[-1] = 1.0, 1.0 / cond
    A = (Q * s) @ Q.T
    return (A + A.T) / 2


def _cw_berr(A, X, B):
    X2 = X.reshape(A.shape[0], -1)
    B2 = B.reshape(A.shape[0], -1)
    R = B2 - A @ X2
    den = np.abs(A) @ np.abs(X2) + np.abs(B2)
    with np.errstate(divide="ignore", invalid="ignore"):
        q = np.where(den > 0, np.abs(R) / den, np.where(R == 0, 0.0, np.inf))
    return float(q.max())


@pytest.mark.parametrize("n,cond", [(300, None), (1000, 1e4), (2048, 1e6), (1500, 1e2)])
def test_mixed_cholesky_fp32_matches_oracle(pkg, oracle, n, cond):
    rng = np.random.default_rng(n)
    A = _spd(rng, n, cond)
    b = rng.standard_normal(n)
    r = pkg.mixed_solve(A, b, maxiter=20, rtol=1e-13, precision="fp32", factorization="cholesky")
    ro = oracle.mixed_solve_chol(A, b, maxiter=20, rtol=1e-13)
    assert r["converged"] and ro["converged"]
    assert not r["fallback"] and not ro["fallback"]
    assert r["factorization"] == "cholesky"
    x = r["x"].cpu().numpy()
    assert _cw_berr(A, x, b) <= 1e-13
    assert abs(r["iterations"] - ro["iterations"]) <= 1
    k = 1.0 if cond is None else cond
    assert np.linalg.norm(x - ro["x"]) <= 100 * k * 1e-13 * np.linalg.norm(ro["x"])


@pytest.mark.parametrize("prec,refine", [("fp16x3", "ir"), ("bf16x3", "auto"), ("fp16", "gmres"), ("bf16", "auto")])
def test_mixed_cholesky_tensor_core_precisions(pkg, prec, refine):
    rng = np.random.default_rng(7)
    n = 2048
    A = _spd(rng, n, 1e4)
    B = rng.standard_normal((n, 3))
    r = pkg.mixed_solve(A, B, maxiter=40, rtol=1e-13, precision=prec, refine=refine, factorization="cholesky")
    assert r["converged"], (prec, refine, r["backward_error"], r["iterations"])
    assert _cw_berr(A, r["x"].cpu().numpy(), B) <= 1e-13


def test_mixed_cholesky_many_rhs_and_normwise(pkg):
    rng = np.random.default_rng(11)
    n = 700
    A = _spd(rng, n, 1e3)
    B = rng.standard_normal((n, 20))  # two chunks of right-hand sides
    r = pkg.mixed_solve(A, B, maxiter=20, rtol=1e-14, precision="fp32", normwise=True, factorization="cholesky")
    assert r["converged"]
    X = r["x"].cpu().numpy()
    R = B - A @ X
    nw = (np.abs(R).max(axis=0) / (np.abs(A).sum(axis=1).max() * np.abs(X).max(axis=0) + np.abs(B).max(axis=0))).max()
    assert nw <= 1e-14


def test_mixed_cholesky_fallback_and_not_posdef(pkg, oracle):
    rng = np.random.default_rng(5)
    n = 100
    A = _spd(rng, n)
    A /= np.abs(A).max()
    # a 2 x 2 block positive definite in Float64 but singular once rounded to Float32
    d = 2.0 ** -30
    A[:2, :] = 0.0
    A[:, :2] = 0.0
    A[0, 0], A[1, 1], A[0, 1], A[1, 0] = 1.0, 1.0, 1.0 - d, 1.0 - d
    b = rng.standard_normal(n)
    r = pkg.mixed_solve(A, b, maxiter=20, rtol=1e-13, precision="fp32", factorization="cholesky")
    ro = oracle.mixed_solve_chol(A, b, maxiter=20, rtol=1e-13)
    assert r["fallback"] and ro["fallback"]
    assert r["reason"] == "working_factor_fallback"
    assert r["converged"] == ro["converged"]
    if r["converged"]:
        assert _cw_berr(A, r["x"].cpu().numpy(), b) <= 1e-13
    with pytest.raises(pkg.PosDefException):
        pkg.mixed_solve(A, b, precision="fp32", factorization="cholesky", fallback=False)
    N = _spd(rng, 50)
    N[20, 20] = -5.0
    with pytest.raises(pkg.PosDefException) as e:
        pkg.mixed_solve(N, np.ones(50), precision="fp32", factorization="cholesky")
    with pytest.raises(ValueError) as eo:
        oracle.mixed_solve_chol(N, np.ones(50))
    assert f"PosDefException({e.value.info})" in str(eo.value)
    with pytest.raises(pkg.ArgumentError):
        pkg.mixed_solve(A, b, factorization="qr")
