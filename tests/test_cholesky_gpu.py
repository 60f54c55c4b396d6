"""Cholesky on the GPU (oxi_dpotrf / oxi_dpotrs) against the oracle's
restatement of cholesky_factor (src/lapack/factorizations.jl:205-305) and the
reference's properties (test/lapack/factorizations.jl style: L L^T = A to
30 n eps, PosDefException on the first failing column, issuccess with
check=false, logabsdet)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
EPS = np.finfo(float).eps


def _np(t):
    return t.detach().cpu().numpy()


def _spd(rng, n, cond=None):
    if cond is None:
        G = rng.standard_normal((n, n))
        return G @ G.T + n * np.eye(n)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = 10.0 ** (-np.log10(cond) * rng.uniform(0, 1, n))
    s[0], s[-1] = 1.0, 1.0 / cond
    A = (Q * s) @ Q.T
    return (A + A.T) / 2


@pytest.mark.parametrize("n", [1, 7, 64, 127, 128, 129, 300, 1000, 2049])
def test_cholesky_matches_oracle(pkg, oracle, n):
    rng = np.random.default_rng(n)
    A = _spd(rng, n)
    F = pkg.cholesky(A)
    assert F.issuccess() and F.info == 0
    L = _np(F.L)
    Lo, info = oracle.potrf(A)
    assert info == 0
    assert np.linalg.norm(L - Lo) / np.linalg.norm(Lo) <= 1e-13
    assert np.linalg.norm(L @ L.T - A) / (np.linalg.norm(A) * n * EPS) <= 30
    assert np.all(np.triu(_np(F.factors), 1) == 0)  # strict upper triangle zeroed
    b = rng.standard_normal(n)
    x = _np(F.solve(torch.from_numpy(b)))
    xo = oracle.potrs(Lo, b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-12
    la, s = F.logabsdet()
    assert s == 1.0 and abs(la - np.linalg.slogdet(A)[1]) <= 1e-10 * max(1.0, abs(la))


def test_cholesky_large_conditioned_and_multi_rhs(pkg, oracle):
    rng = np.random.default_rng(3)
    n = 6000
    A = _spd(rng, n, cond=1e6)
    F = pkg.cholesky(A)
    L = _np(F.L)
    assert np.linalg.norm(L @ L.T - A) / (np.linalg.norm(A) * n * EPS) <= 30
    B = rng.standard_normal((n, 5))
    X = _np(F.solve(torch.from_numpy(B)))
    R = B - A @ X
    assert np.abs(R).max() / (np.abs(A).max() * np.abs(X).max() * n) <= 30 * EPS


def test_cholesky_failures_and_in_place(pkg, oracle):
    rng = np.random.default_rng(4)
    n = 300
    A = _spd(rng, n)
    A[200, 200] = -1.0  # the leading minor of order 201 is not positive definite
    with pytest.raises(pkg.PosDefException) as e:
        pkg.cholesky(A)
    _, info_o = oracle.potrf(A)
    assert e.value.info == info_o
    F = pkg.cholesky(A, check=False)
    assert not F.issuccess() and F.info == info_o
    with pytest.raises(pkg.PosDefException):
        F.solve(np.ones(n))
    N = rng.standard_normal((5, 5))  # not symmetric
    with pytest.raises(pkg.PosDefException) as e:
        pkg.cholesky(N)
    assert e.value.info == -1
    assert pkg.cholesky(N, check=False).info == -1
    # cholesky!: the lower triangle in place, only it is read
    B = _spd(rng, 150)
    M = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()  # memory = B column-major
    Acm = M.t()
    with torch.no_grad():
        Acm[np.triu_indices(150, 1)] = 7.0  # the upper triangle is not read
    G = pkg.cholesky_(Acm)
    Lo, _ = oracle.potrf(B)
    assert np.linalg.norm(_np(Acm) - Lo) / np.linalg.norm(Lo) <= 1e-13
    assert np.linalg.norm(_np(G.L) - Lo) / np.linalg.norm(Lo) <= 1e-13


@pytest.mark.parametrize("ld_extra", [0, 7])
def test_cholesky_inplace_failure_keeps_upper_triangle(pkg, oracle, ld_extra):
    """cholesky!(A; check=false) on a matrix that is not positive definite:
    info is the failing column and the strict upper triangle (not read, and
    not zeroed on failure) is left as it was, also for an odd leading
    dimension (a view, linalg_api.jl:54-76)."""
    rng = np.random.default_rng(40 + ld_extra)
    n = 300
    A = _spd(rng, n)
    A[200, 200] = -1.0
    _, info_o = oracle.potrf(A)
    ld = n + ld_extra
    big = torch.zeros((n, ld), dtype=torch.float64, device="cuda")  # memory: column-major n x n, leading dim ld
    Acm = big.t()[:n, :]
    assert Acm.stride(0) == 1 and Acm.stride(1) == ld
    with torch.no_grad():
        Acm.copy_(torch.from_numpy(A))
        iu = np.triu_indices(n, 1)
        Acm[iu] = 5.0
    G = pkg.cholesky_(Acm, check=False)
    assert not G.issuccess() and G.info == info_o == 201
    assert np.all(_np(Acm)[iu] == 5.0)
    # and the successful in-place factorization with the odd leading dimension
    B = _spd(rng, n)
    with torch.no_grad():
        Acm.copy_(torch.from_numpy(B))
    G = pkg.cholesky_(Acm)
    Lo, _ = oracle.potrf(B)
    assert np.linalg.norm(_np(G.L) - Lo) / np.linalg.norm(Lo) <= 1e-13
    assert np.all(np.triu(_np(Acm), 1) == 0)


@pytest.mark.parametrize("n", [700, 2049])
def test_cholesky_lookahead_gives_identical_factor(pkg, n):
    """The lookahead (next block's rows first, the rest of the symmetric update
    on a second stream) changes only the schedule: the same factor, bit for bit."""
    rng = np.random.default_rng(n + 5)
    A = _spd(rng, n, cond=1e5)
    with pkg.options(lookahead=0):
        L0 = _np(pkg.cholesky(A).L)
    with pkg.options(lookahead=1):
        L1 = _np(pkg.cholesky(A).L)
    assert np.array_equal(L0, L1)
