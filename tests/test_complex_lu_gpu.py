"""GPU parity of the complex (ComplexF64) dense LU against the oracle.

The API cases follow test/api/linalg_api.jl:22-76 ("dense LU $T" and
"in-place lu!/cholesky! on views $T" for ComplexF64).  Against the oracle
(orc_zgetrf, a restatement of _lu_factor! / _lu_panel! for complex types):
pivot sequences identical; factors within 1e-11 relative and solves within
1e-10 relative of the oracle's on the same factors (the GPU forms each complex
product as four real products on the FP64 tensor cores, the oracle as one
complex multiply-add chain, so the last bits differ); normwise backward
error of P A = L U <= 30 (units of eps * n, test/lapack/lapack_dense.jl:4).
"""
import numpy as np
import pytest
import torch

from conftest import bwd

pytestmark = pytest.mark.gpu
RT = 1e-8  # _api_rt(ComplexF64), test/api/linalg_api.jl:7


def _np(t):
    return t.detach().cpu().numpy()


def _crandn(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _close(x, y, rtol=RT):
    x, y = np.asarray(x), np.asarray(y)
    return np.linalg.norm(x - y) <= rtol * max(np.linalg.norm(x), np.linalg.norm(y))


def _split(F, m, n):
    q = min(m, n)
    return np.tril(F[:, :q], -1) + np.eye(m, q), np.triu(F[:q, :])


def test_dense_lu_api_complex(pkg):
    rng = np.random.default_rng(9)
    n = 9
    A = _crandn(rng, n, n)
    b = _crandn(rng, n)
    B = _crandn(rng, n, 3)
    F = pkg.lu(A)
    assert F.shape == (n, n) and F.issuccess() and F.dtype == torch.complex128
    L, U, p = _np(F.L), _np(F.U), F.p
    assert _close(L @ U, A[p, :])
    assert _close(_np(F.P) @ A, L @ U)
    assert _close(_np(F.solve(b)), np.linalg.solve(A, b))
    assert _close(_np(F.solve(B)), np.linalg.solve(A, B))
    assert _close(_np(F.H.solve(b)), np.linalg.solve(A.conj().T, b))
    assert _close(_np(F.T.solve(b)), np.linalg.solve(A.T, b))
    Bt = torch.as_tensor(B, device="cuda").clone()
    assert _close(_np(F.ldiv_(Bt)), np.linalg.solve(A, B))
    y = torch.empty(n, dtype=torch.complex128, device="cuda")
    assert _close(_np(pkg.ldiv_into(y, F, b)), np.linalg.solve(A, b))
    assert np.isclose(F.det(), np.linalg.det(A), rtol=RT)
    assert np.isclose(pkg.det(A), np.linalg.det(A), rtol=RT)
    sgn, la = np.linalg.slogdet(A)
    la2, s2 = pkg.logabsdet(A)
    assert np.isclose(la2, la, rtol=RT) and np.isclose(s2, sgn, rtol=RT)
    assert _close(_np(pkg.inv(F)), np.linalg.inv(A))
    assert _close(_np(pkg.inv(A)), np.linalg.inv(A))
    bi = np.round(b.real).astype(np.int64)  # F \ Int.(round.(real.(b)))
    assert _close(_np(F.solve(bi)), np.linalg.solve(A, bi))
    S = A.copy()
    S[:, 1] = 0
    G = pkg.lu(S, check=False)
    assert not G.issuccess()
    with pytest.raises(pkg.SingularException):
        G.solve(b)
    with pytest.raises(pkg.SingularException):
        pkg.lu(S)
    assert G.det() == 0
    assert F.propertynames() == ("L", "U", "p", "P")


@pytest.mark.parametrize("n", [9, 300])
def test_lu_inplace_on_views_complex(pkg, n):
    """lu!(X) on a plain matrix, on a view with leading dimension > m, and on
    a view with row stride 2 (linalg_api.jl:54-66)."""
    rng = np.random.default_rng(n)
    b = _crandn(rng, n)
    # column-major Big (n+7) x (n+5): the torch tensor (n+5, n+7) transposed
    big_t = torch.as_tensor(_crandn(rng, n + 5, n + 7), device="cuda")
    Big = big_t.t()
    outside = Big.clone()
    V = Big[3:n + 3, 2:n + 2]
    assert V.stride(0) == 1 and V.stride(1) == n + 7
    big2 = torch.as_tensor(_crandn(rng, 2 * n, n), device="cuda")
    W = big2[0::2, :]
    Xp = torch.as_tensor(_crandn(rng, n, n), device="cuda")
    for X in (Xp, V, W):
        A = _np(X).copy()
        F = pkg.lu_(X)
        if X.stride(0) == 1:
            assert F.factors is X
        assert _close(_np(F.solve(b)), np.linalg.solve(A, b))
        L, U = _np(F.L), _np(F.U)
        assert _close(L @ U, A[F.p, :])
        assert bwd(L @ U - A[F.p, :], A) <= 30
    after = _np(Big)
    ref = _np(outside)
    assert np.array_equal(after[:3, :], ref[:3, :])
    assert np.array_equal(after[:, :2], ref[:, :2])
    S = torch.as_tensor(_crandn(rng, 6, 6), device="cuda").t().contiguous().t()
    S[:, 2] = 0
    F = pkg.lu_(S, check=False)
    assert not F.issuccess() and F.factors is S


@pytest.mark.parametrize("m,n,bs", [(64, 64, 128), (300, 300, 128), (1000, 1000, 128), (2048, 2048, 128),
                                    (500, 300, 128), (300, 500, 128), (777, 777, 100), (1500, 1500, 64),
                                    (900, 900, 256), (9000, 64, 128), (13000, 48, 128)])
def test_complex_pivots_and_factors_vs_oracle(pkg, oracle, m, n, bs):
    rng = np.random.default_rng(m * 7 + n + bs)
    A = _crandn(rng, m, n)
    F = pkg.lu(A, blocksize=bs, check=False)
    Fo, ipo, info = oracle.zgetrf(A, blocksize=bs)
    assert F.info == info == 0
    assert np.array_equal(_np(F.ipiv), ipo)
    fac = _np(F.factors)
    assert np.linalg.norm(fac - Fo) <= 1e-11 * np.linalg.norm(Fo)
    L, U = _split(fac, m, n)
    assert bwd(L @ U - A[F.p, :], A) <= 30


@pytest.mark.parametrize("trans", ["N", "T", "C"])
def test_complex_solves_vs_oracle(pkg, oracle, trans):
    rng = np.random.default_rng(ord(trans))
    n = 700
    A = _crandn(rng, n, n)
    B = _crandn(rng, n, 5)
    F = pkg.lu(A)
    fac, ipiv = _np(F.factors), _np(F.ipiv)
    Xo = oracle.zgetrs(fac, ipiv, B, trans)  # the oracle solve with the GPU's factors
    G = {"N": F, "T": F.T, "C": F.H}[trans]
    X = _np(G.solve(B))
    assert np.linalg.norm(X - Xo) <= 1e-10 * np.linalg.norm(Xo)
    M = {"N": A, "T": A.T, "C": A.conj().T}[trans]
    r = np.linalg.norm(M @ X - B) / (np.linalg.norm(M) * np.linalg.norm(X) * n * np.finfo(float).eps)
    assert r <= 30


def test_complex_pivot_rule_overflow_and_nan(pkg, oracle):
    """abs2 overflows -> the scan is redone with abs; a NaN on the diagonal
    keeps row j (the strict '>' against a NaN start, factorizations.jl:92-107)."""
    rng = np.random.default_rng(5)
    n = 40
    A = _crandn(rng, n, n)
    A[7, 0] = 3e200 + 1e200j  # abs2 overflows
    A[11, 0] = 1e200 - 3.1e200j  # larger modulus, abs2 also infinite
    F = pkg.lu(A, check=False)
    Fo, ipo, info = oracle.zgetrf(A)
    assert np.array_equal(_np(F.ipiv), ipo)
    assert ipo[0] == 12
    B = _crandn(rng, n, n)
    B[0, 0] = complex(np.nan, 1.0)
    B[5, 0] = 100.0
    G = pkg.lu(B, check=False)
    Go, ipg, _ = oracle.zgetrf(B)
    assert _np(G.ipiv)[0] == ipg[0] == 1
    assert np.array_equal(_np(G.ipiv), ipg)


def test_complex_singular_info_and_empty(pkg, oracle):
    rng = np.random.default_rng(3)
    A = _crandn(rng, 200, 200)
    A[:, 37] = 0
    F = pkg.lu(A, check=False)
    _, _, info = oracle.zgetrf(A)
    assert F.info == info == 38
    E = pkg.lu(np.zeros((0, 0), dtype=np.complex128))
    assert E.shape == (0, 0) and E.issuccess()
