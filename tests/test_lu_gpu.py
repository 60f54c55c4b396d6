"""GPU parity of the dense LU path against the oracle and LAPACK golden vectors.

Bars: pivot sequences identical; factors bit-identical to the oracle (FP64,
both the tensor-core engine and the reference-order mode); normwise
backward error <= 30 (units of eps * max(m, n), test/lapack/lapack_dense.jl:4);
solve backward error <= 30 * cond(A) (lapack_dense.jl:15-20).
"""
import numpy as np
import pytest
import scipy.linalg as sl
import torch

from conftest import bwd, entry_oracle, split_lu

pytestmark = pytest.mark.gpu
NEAR_TIES = ("singular", "nearly_singular")


def _np(t):
    return t.detach().cpu().numpy()


def test_golden_cases_tensor_engine(pkg, oracle, golden):
    for name, c in golden.items():
        A = c["A"]
        m, n = A.shape
        F = pkg.lu(A, check=False, blocksize=c["bs"])
        fac = _np(F.factors)
        ipiv = _np(F.ipiv)
        Fo, ipo, info = oracle.getrf(A, blocksize=c["bs"], check=False)
        assert F.info == info == c["info"], name
        assert np.array_equal(ipiv, ipo), name
        if not name.startswith(NEAR_TIES):
            assert np.array_equal(ipiv, c["ipiv"]), name
        # FP64: the tensor-core engine's operations are the reference's, in
        # the reference's order -- the same bits
        assert np.array_equal(fac, Fo), name
        L, U = split_lu(fac, m, n)
        assert bwd(L @ U - A[F.p, :], A) <= 30, name


def test_golden_cases_reference_order_bit_identical(pkg, oracle, golden):
    with pkg.options(gemm="reference", trsm_leaf=8):
        for name, c in golden.items():
            A = c["A"]
            F = pkg.lu(A, check=False, blocksize=c["bs"])
            Fo, ipo, info = oracle.getrf(A, blocksize=c["bs"], check=False)
            assert np.array_equal(_np(F.ipiv), ipo), name
            assert np.array_equal(_np(F.factors), Fo), name


@pytest.mark.parametrize("n,bs", [(600, 128), (1024, 128), (2048, 128), (1000, 100), (777, 64)])
def test_randn_pivots_and_factors(pkg, oracle, n, bs):
    rng = np.random.default_rng(n + bs)
    A = rng.standard_normal((n, n))
    F = pkg.lu(A, blocksize=bs)
    Fo, ipo, _ = oracle.getrf(A, blocksize=bs)
    assert np.array_equal(_np(F.ipiv), ipo)
    assert np.array_equal(_np(F.factors), Fo)
    _, piv = sl.lu_factor(A)
    assert np.array_equal(_np(F.ipiv), piv + 1)  # == LAPACK getrf


@pytest.mark.parametrize("m,n", [(9000, 300), (17000, 100), (17000, 200)])
def test_tall_panel_leaf_widths(pkg, m, n):
    """m > 8192 rows switches the FP64 leaf kernel to 16 columns, m > 16384 to
    8: the 32-column leaf is emulated (in a composed panel, n > 128, and in a
    single narrow panel)."""
    rng = np.random.default_rng(9)
    A = rng.standard_normal((m, n))
    F = pkg.lu(A)
    _, piv = sl.lu_factor(A)
    assert np.array_equal(_np(F.ipiv), piv[:n] + 1)
    # the 16-column leaves plus the in-order rank-16 steps give the 32-column
    # leaf's bits
    Fo, _, _ = entry_oracle().getrf(A)
    assert np.array_equal(_np(F.factors), Fo)
    L, U = split_lu(_np(F.factors), m, n)
    assert bwd(L @ U - A[F.p, :], A) <= 30


def test_singular_and_check(pkg, golden):
    A = golden["singular_col23_40"]["A"]
    with pytest.raises(pkg.SingularException) as e:
        pkg.lu(A)
    assert e.value.info == 23
    F = pkg.lu(A, check=False)
    assert F.info == 23 and not F.issuccess()
    with pytest.raises(pkg.SingularException):
        F.solve(np.ones(40))
    Z = pkg.lu(np.zeros((3, 3)), check=False)
    assert Z.info == 1


def test_lu_inplace_column_major_and_views(pkg):
    rng = np.random.default_rng(1)
    for n in (9, 300):
        b = torch.from_numpy(rng.standard_normal(n)).cuda()
        X = torch.from_numpy(rng.standard_normal((n, n))).cuda().t().contiguous().t()  # column-major
        A = X.clone()
        F = pkg.lu_(X)
        assert F.factors.data_ptr() == X.data_ptr()
        x = pkg.ldiv(F, b)
        assert torch.allclose(A @ x, b, rtol=1e-10, atol=1e-10)
        # strided view with leading dimension > m (a Julia view(Big, 4:n+3, 3:n+2))
        Big = torch.from_numpy(rng.standard_normal((n + 5, n + 7))).cuda().t()  # (n+7, n+5)^T storage
        Bigc = Big.clone()
        V = Big[3:n + 3, 2:n + 2]
        assert V.stride(0) == 1
        Av = V.clone()
        F = pkg.lu_(V)
        L, U = split_lu(_np(F.factors), n, n)
        assert bwd(L @ U - _np(Av)[F.p, :], _np(Av)) <= 30
        mask = torch.ones_like(Big, dtype=torch.bool)
        mask[3:n + 3, 2:n + 2] = False
        assert torch.equal(Big[mask], Bigc[mask])
        # row-major input: factored through a copy, factors written back
        R = torch.from_numpy(rng.standard_normal((n, n))).cuda()
        Ar = R.clone()
        F = pkg.lu_(R)
        assert torch.equal(R, F.factors)
        L, U = split_lu(_np(R), n, n)
        assert bwd(L @ U - _np(Ar)[F.p, :], _np(Ar)) <= 30


def test_solves_match_reference_api(pkg):
    """test/api/linalg_api.jl:23-52 on the GPU engine."""
    rng = np.random.default_rng(2)
    for n in (9, 130, 1000):
        A = rng.standard_normal((n, n))
        b = rng.standard_normal(n)
        B = rng.standard_normal((n, 3))
        F = pkg.lu(A)
        r = 1e-9 if n < 1000 else 1e-8
        ref = np.linalg.solve(A, b)
        assert np.allclose(_np(F.solve(b)), ref, rtol=r, atol=r)
        assert np.allclose(_np(pkg.ldiv(F, B)), np.linalg.solve(A, B), rtol=r, atol=r)
        assert np.allclose(_np(pkg.ldiv(F.T, b)), np.linalg.solve(A.T, b), rtol=r, atol=r)
        assert np.allclose(_np(pkg.ldiv(F.H, b)), np.linalg.solve(A.T, b), rtol=r, atol=r)
        Bt = torch.from_numpy(B.copy()).cuda()
        out = pkg.ldiv_(F, Bt)
        assert out is Bt and np.allclose(_np(Bt), np.linalg.solve(A, B), rtol=r, atol=r)
        Y = torch.empty(n, dtype=torch.float64, device="cuda")
        bt = torch.from_numpy(b).cuda()
        assert pkg.ldiv_into(Y, F, bt) is Y and torch.equal(bt.cpu(), torch.from_numpy(b))
        bc = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.allclose(_np(pkg.ldiv(F, bc)), np.linalg.solve(A, bc), rtol=r, atol=r)
        bi = np.round(b).astype(np.int64)
        assert np.allclose(_np(pkg.ldiv(F, bi)), np.linalg.solve(A, bi), rtol=r, atol=r)
        c = np.linalg.cond(A)
        X = _np(pkg.ldiv(F, B))
        assert bwd(A @ X - B, A) <= 30 * c
        assert np.isclose(F.det(), np.linalg.det(A), rtol=1e-9)
        la, s = F.logabsdet()
        sa, laa = np.linalg.slogdet(A)
        assert np.isclose(la, laa, rtol=1e-10) and s == sa
        P = _np(F.P)
        assert np.allclose(P @ A, _np(F.L) @ _np(F.U), rtol=1e-10, atol=1e-10)
        assert F.propertynames() == ("L", "U", "p", "P")


def test_gemm_update_matches_torch(pkg):
    torch.manual_seed(0)
    for (m, n, k) in ((1, 1, 1), (127, 65, 128), (300, 500, 128), (1024, 2048, 128), (517, 263, 37),
                      (2000, 64, 256), (64, 3000, 16)):
        A = torch.randn(m, k, dtype=torch.float64, device="cuda")
        B = torch.randn(k, n, dtype=torch.float64, device="cuda")
        C = torch.randn(m, n, dtype=torch.float64, device="cuda")
        ref = C - A @ B
        pkg.gemm_update(C, A, B)
        err = (C - ref).abs().max().item() / max(1.0, ref.abs().max().item())
        assert err <= 1e-13, (m, n, k, err)


def test_float32_lu(pkg, oracle):
    rng = np.random.default_rng(4)
    for n in (64, 300, 1500):
        A = rng.standard_normal((n, n)).astype(np.float32)
        F = pkg.lu(torch.from_numpy(A))
        Fo, ipo, _ = oracle.getrf(A, dtype=np.float32)
        assert np.array_equal(_np(F.ipiv), ipo)
        L, U = split_lu(_np(F.factors).astype(np.float64), n, n)
        assert bwd(L @ U - A[F.p, :].astype(np.float64), A) <= 30
        b = rng.standard_normal(n).astype(np.float32)
        x = _np(F.solve(torch.from_numpy(b)))
        assert np.linalg.norm(A @ x - b) / (np.linalg.norm(A) * np.linalg.norm(x)) < 1e-5


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_transposed_solve_unaligned_leading_dimension(pkg, dtype):
    """ldiv!(transpose(F), B) when lda * sizeof(T) is not a multiple of 16: the
    transposed triangular solves read the factor along rows, so their row
    starts are not 16-byte aligned (n = 331, 333 odd; n = 258 for FP32)."""
    rng = np.random.default_rng(6)
    for n in (258, 331, 333):
        A = (rng.standard_normal((n, n)) + 4 * np.eye(n)).astype(dtype)
        B = rng.standard_normal((n, 3)).astype(dtype)
        F = pkg.lu(torch.from_numpy(A))
        r = 1e-9 if dtype == np.float64 else 2e-3
        ref64 = A.astype(np.float64)
        for Fv, M in ((F, ref64), (F.T, ref64.T), (F.H, ref64.T)):
            X = _np(pkg.ldiv(Fv, torch.from_numpy(B))).astype(np.float64)
            assert np.allclose(X, np.linalg.solve(M, B.astype(np.float64)), rtol=r, atol=r), (n, dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_lookahead_gives_identical_factors(pkg, oracle, dtype):
    """OXI_OPT_LOOKAHEAD on or off leaves getrf's pivots and factors bit-identical
    (for FP64 and native FP32 the option keeps the plain schedule), and the
    pivots match the oracle's."""
    rng = np.random.default_rng(41)
    for n, bs in ((1000, 128), (1537, 64)):
        A = rng.standard_normal((n, n)).astype(dtype)
        with pkg.options(lookahead=0):
            F0 = pkg.lu(torch.from_numpy(A), blocksize=bs)
        with pkg.options(lookahead=1):
            F1 = pkg.lu(torch.from_numpy(A), blocksize=bs)
        assert torch.equal(F0.ipiv, F1.ipiv)
        assert torch.equal(F0.factors, F1.factors)
        if dtype == np.float64:
            _, ipo, _ = oracle.getrf(A, blocksize=bs)
            assert np.array_equal(_np(F1.ipiv), ipo)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_many_rhs_solves_every_chunk_width(pkg, dtype):
    """ldiv! with 23 right-hand sides runs the block-operator triangular solve
    in chunks of 16 (FP32), 8, 4, 2 and 1 columns; n = 777 gives a partial last
    64-row block and more blocks than the three the chain couples.  Each column
    must equal the one-column solve of the same factor (relative 1e-13 FP64,
    1e-5 FP32: the per-column arithmetic does not depend on the chunk width),
    and the whole solve must have a normwise backward error <= 30 n eps, for N
    and T."""
    rng = np.random.default_rng(77)
    n, k = 777, 23
    A = (rng.standard_normal((n, n)) + 4 * np.eye(n)).astype(dtype)
    B = rng.standard_normal((n, k)).astype(dtype)
    F = pkg.lu(torch.from_numpy(A))
    same = 1e-13 if dtype == np.float64 else 1e-5
    eps = np.finfo(dtype).eps
    A64, B64 = A.astype(np.float64), B.astype(np.float64)
    for Fv, M in ((F, A64), (F.T, A64.T)):
        X = _np(pkg.ldiv(Fv, torch.from_numpy(B))).astype(np.float64)
        for j in (0, 7, 15, 16, 22):
            xj = _np(pkg.ldiv(Fv, torch.from_numpy(np.ascontiguousarray(B[:, j])))).astype(np.float64)
            assert np.abs(X[:, j] - xj).max() <= same * np.abs(xj).max(), (dtype, j)
        bw = np.linalg.norm(M @ X - B64) / (np.linalg.norm(M) * np.linalg.norm(X))
        assert bw <= 30 * n * eps, (dtype, bw)


@pytest.mark.parametrize("m,n", [(300, 300), (9000, 64)])
def test_nan_pivot_rule_matches_oracle(pkg, oracle, m, n):
    """_lu_pivot (src/lapack/factorizations.jl:92-107) starts from row j with a
    strict '>': a NaN at row j keeps row j although larger finite rows lie
    below; a NaN below the diagonal never wins.  The GPU leaf follows it, so
    the pivots (and the bits) equal the oracle's."""
    rng = np.random.default_rng(m + n)
    A = rng.standard_normal((m, n))
    A[5, 5] = np.nan          # column 5: row 5 kept
    A[40, 2] = np.nan         # column 2: never the pivot
    F = pkg.lu(A, check=False)
    Fo, ipo, _ = oracle.getrf(A, check=False)
    ipiv = _np(F.ipiv)
    assert ipiv[5] == 6
    assert np.array_equal(ipiv, ipo)
    assert np.array_equal(_np(F.factors), Fo, equal_nan=True)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.complex128])
def test_layout_copy_on_the_engine(pkg, dtype):
    """colmajor_copy runs oxi_transpose (the engine's tiled transpose) for
    contiguous row-major inputs: the column-major copy equals torch's."""
    g = torch.Generator(device="cuda").manual_seed(3)
    for m, n in ((1, 1), (33, 65), (1000, 7), (640, 1031)):
        if dtype.is_complex:
            t = torch.complex(torch.randn(m, n, generator=g, device="cuda", dtype=torch.float64),
                              torch.randn(m, n, generator=g, device="cuda", dtype=torch.float64))
        else:
            t = torch.randn(m, n, generator=g, device="cuda", dtype=dtype)
        out = pkg.colmajor_copy(t)
        assert out.shape == (n, m)
        assert torch.equal(out, t.t().contiguous())
