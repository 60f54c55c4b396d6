"""Parity at the benchmarked configurations (the sizes the benchmark reports).

- Plain FP64 LU at n = 8192 and at the headline n = 16384 on the kappa ~ 1e4
  construction (U diag(sigma) V^T, sigma log-uniform): pivots identical to the
  oracle's (which restates _lu_factor!, src/lapack/factorizations.jl:30-77),
  factors bit-identical to the oracle's, normwise backward error of
  L U - A[p, :] <= 30 (units of eps * n, test/lapack/lapack_dense.jl:4).
- The plain path as the reference benchmarks it: randn(1024) + 1024 I, one
  right-hand side (benchmark/suite/inputs.jl:109-110).
- The mixed solve with 16 right-hand sides at n = 8192, kappa 1e4.
- The badly scaled construction (kappa 1e6, rows scaled by 10^U(-3,3)) at
  n = 8192 through split FP16 with AUTO refinement and with GMRES-IR.
- The GPU equilibration against equilibrate(A; radix=true), exactly.
Every backward error is the oracle's (FP64 on the host).
"""
import numpy as np
import pytest
import torch

from conftest import bwd, split_lu

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("n", [8192, 16384])
def test_plain_fp64_lu_at_benchmark_sizes(pkg, oracle, n):
    A = pkg.synthetic.kappa_matrix(n, 1e4, seed=20261104)
    F = pkg.lu(A)
    ipiv = _np(F.ipiv)
    Fo, ipo, info = oracle.getrf(_np(A))
    assert info == 0
    assert np.array_equal(ipiv, ipo), int(np.argmax(ipiv != ipo))
    fac = F.factors
    # the FP64 engine performs the reference's operations in the reference's
    # order (DMMA fma chains, the recursive TRSM's steps, the 32-column leaf's
    # rank-1 steps): the factors are the same bits
    assert np.array_equal(_np(fac), Fo), np.linalg.norm(_np(fac) - Fo) / np.linalg.norm(Fo)
    del Fo
    # backward error of the GPU factors (the product L U formed by torch in FP64
    # as a checker): ||L U - A[p, :]||_F / (||A||_F n eps)
    p = torch.from_numpy(oracle.perm_from_ipiv(ipiv, n)).cuda()
    E = torch.tril(fac, -1)
    E.diagonal().fill_(1.0)
    E = E @ torch.triu(fac)
    E -= A[p, :]
    e = (torch.linalg.norm(E) / (torch.linalg.norm(A) * n * np.finfo(float).eps)).item()
    assert e <= 30, e


def test_plain_config_randn_plus_nI_one_rhs(pkg, oracle):
    """A = randn(1024,1024) + 1024 I (seeded PCG64), b = randn(1024): pivots,
    factors and ||Ax - b|| / (||A|| ||x||) against the oracle."""
    rng = np.random.Generator(np.random.PCG64(20261104))
    n = 1024
    A = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal(n)
    F = pkg.lu(A)
    Fo, ipo, info = oracle.getrf(A)
    assert info == 0 and np.array_equal(_np(F.ipiv), ipo)
    assert np.array_equal(_np(F.factors), Fo)
    x = _np(pkg.ldiv(F, torch.from_numpy(b)))
    xo = oracle.getrs(Fo, ipo, b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-13
    r = np.linalg.norm(A @ x - b) / (np.linalg.norm(A) * np.linalg.norm(x))
    assert r <= 30 * n * np.finfo(float).eps, r
    assert oracle.normwise_backward_error(A, x, b) <= 1e-15


def test_mixed_16rhs_n8192_kappa1e4(pkg, oracle):
    n, nrhs = 8192, 16
    A = pkg.synthetic.kappa_matrix(n, 1e4, seed=20261105)
    g = torch.Generator(device="cuda").manual_seed(20261106)
    B = torch.randn(n, nrhs, dtype=torch.float64, device="cuda", generator=g)
    r = pkg.mixed_solve(A, B, precision="fp16x3", refine="auto", rtol=1e-14, normwise=True, maxiter=30)
    assert r["converged"], {k: v for k, v in r.items() if k != "x"}
    An, Bn, X = _np(A), _np(B), _np(r["x"])
    for k in range(nrhs):
        assert oracle.normwise_backward_error(An, X[:, k], Bn[:, k]) <= 1e-14, k
    # forward error against the plain FP64 GPU solve: within kappa * 1e-13
    F = pkg.lu(A)
    Xp = _np(pkg.ldiv(F, B))
    fe = np.linalg.norm(X - Xp) / np.linalg.norm(Xp)
    assert fe <= 1e4 * 1e-13, fe


@pytest.mark.parametrize("prec,refine", [("fp16x3", "auto"), ("fp16x3", "gmres")])
def test_mixed_badly_scaled_kappa1e6_n8192(pkg, oracle, prec, refine):
    """kappa 1e6 with rows scaled by 10^U(-3,3): the equilibration and the FP16
    power-of-two operand scaling must keep every converted value finite."""
    n = 8192
    A = pkg.synthetic.kappa_matrix(n, 1e6, seed=20261107, row_scale_decades=3.0)
    g = torch.Generator(device="cuda").manual_seed(20261108)
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    r = pkg.mixed_solve(A, b, precision=prec, refine=refine, rtol=1e-14, normwise=True, maxiter=30)
    assert r["converged"] and not r["fallback"], {k: v for k, v in r.items() if k != "x"}
    An, bn, x = _np(A), _np(b), _np(r["x"])
    assert oracle.normwise_backward_error(An, x, bn) <= 1e-14


def test_gpu_equilibration_matches_oracle_exactly(pkg, oracle):
    rng = np.random.default_rng(31)
    for (m, n) in [(300, 200), (1, 7), (7, 1), (1000, 1000)]:
        A = rng.standard_normal((m, n)) * (10.0 ** rng.uniform(-3, 3, (m, 1)))
        A[0, :] = 0.0  # a zero row keeps scale 1
        if n > 2:
            A[:, 2] = 0.0  # and a zero column
        E = pkg.equilibrate(A)
        Eo, ro, co = oracle.equilibrate_radix(A)
        assert np.array_equal(_np(E["row_scale"]), ro)
        assert np.array_equal(_np(E["column_scale"]), co)
        assert np.array_equal(_np(E["matrix"]), Eo)
    # row maxima at and around the rounding boundary 2^k * sqrt(2) and near
    # the ends of the exponent range
    s2 = np.sqrt(2.0)
    vals = []
    for k in (-1000, -3, 0, 1, 7, 900):
        c = np.ldexp(s2, k)
        vals += [c, np.nextafter(c, 0), np.nextafter(c, np.inf), np.ldexp(1.0, k), np.ldexp(1.5, k)]
    vals += [np.finfo(float).tiny, 5e-324, np.finfo(float).max]
    A = np.array(vals)[:, None] * np.ones((1, 3))
    E = pkg.equilibrate(A)
    _, ro, co = oracle.equilibrate_radix(A)
    assert np.array_equal(_np(E["row_scale"]), ro)
    assert np.array_equal(_np(E["column_scale"]), co)
    # config 5's matrix at n = 8192, the input the mixed solve equilibrates
    A = pkg.synthetic.kappa_matrix(8192, 1e6, seed=20261107, row_scale_decades=3.0)
    E = pkg.equilibrate(A)
    _, ro, co = oracle.equilibrate_radix(_np(A))
    assert np.array_equal(_np(E["row_scale"]), ro)
    assert np.array_equal(_np(E["column_scale"]), co)
    with pytest.raises(pkg.ArgumentError):
        pkg.equilibrate(np.array([[1.0, np.inf]]))
