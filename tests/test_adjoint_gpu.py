"""GPU parity of the reverse-mode rule of x = A \\ b (oxi_dlu_adjoint).

Checks, for loss 0.5 ||x||^2 (xbar = x):
  * against the oracle's adjoint on its own CPU LU (the reference gradient);
  * against central finite differences, h = 1e-6, on 64 random unit directions
    of A and 8 of b, at n = 2048 with kappa = 1e3 (sigma log-uniform on
    [1e-3, 1], Haar U and V);
  * through torch.autograd (solve) against torch.linalg.solve's own gradient;
  * several right-hand sides (two passes of the rank-16 kernel), an odd
    leading dimension of Abar, nrhs = 0, and argument errors.
Tolerances are written in each assertion.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def test_adjoint_matches_oracle(pkg, oracle):
    rng = np.random.default_rng(21)
    for n in (1, 7, 200, 513):
        A = rng.standard_normal((n, n)) + n * np.eye(n) * 0.1
        b = rng.standard_normal(n)
        F = pkg.lu(A)
        x = F.solve(b)
        bbar, Abar = pkg.lu_adjoint(F, x, x)
        Fo, ipo, _ = oracle.getrf(A)
        xo = oracle.getrs(Fo, ipo, b)
        bo, Ao = oracle.lu_adjoint(Fo, ipo, xo, xo)
        sb = np.abs(bo).max()
        sa = np.abs(Ao).max()
        assert np.abs(_np(bbar) - bo).max() <= 1e-10 * sb, n
        assert np.abs(_np(Abar) - Ao).max() <= 1e-10 * sa, n


def test_adjoint_finite_differences_kappa_1e3(pkg, oracle):
    n = 2048
    A = pkg.synthetic.kappa_matrix(n, 1e3, seed=4242)
    g = torch.Generator(device="cuda").manual_seed(4243)
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    F = pkg.lu(A)
    x = F.solve(b)
    bbar, Abar = pkg.lu_adjoint(F, x, x)

    def loss(Am, bv):
        y = pkg.lu(Am).solve(bv)
        return 0.5 * float((y * y).sum())

    h = 1e-6
    na = float(torch.linalg.norm(Abar))
    worst = 0.0
    for _ in range(64):
        D = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        D /= torch.linalg.norm(D)
        fd = (loss(A + h * D, b) - loss(A - h * D, b)) / (2 * h)
        an = float((Abar * D).sum())
        worst = max(worst, abs(fd - an) / na)
    assert worst <= 1e-6, worst  # relative to ||Abar||_F
    nb = float(torch.linalg.norm(bbar))
    for _ in range(8):
        d = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
        d /= torch.linalg.norm(d)
        fd = (loss(A, b + h * d) - loss(A, b - h * d)) / (2 * h)
        assert abs(fd - float((bbar * d).sum())) <= 1e-6 * nb
    # reference gradient from the oracle's CPU LU
    An, bn = _np(A), _np(b)
    Fo, ipo, _ = oracle.getrf(An)
    xo = oracle.getrs(Fo, ipo, bn)
    bo, Ao = oracle.lu_adjoint(Fo, ipo, xo, xo)
    assert np.abs(_np(bbar) - bo).max() <= 1e-9 * np.abs(bo).max()
    assert np.abs(_np(Abar) - Ao).max() <= 1e-9 * np.abs(Ao).max()


def test_autograd_solve_matches_torch(pkg):
    torch.manual_seed(5)
    n = 300
    A0 = torch.randn(n, n, dtype=torch.float64, device="cuda") + 5 * torch.eye(n, device="cuda")
    b0 = torch.randn(n, 3, dtype=torch.float64, device="cuda")
    A1, b1 = A0.clone().requires_grad_(), b0.clone().requires_grad_()
    x1 = pkg.solve(A1, b1)
    (0.5 * (x1 ** 2).sum() + x1[:, 1].sum()).backward()
    A2, b2 = A0.clone().requires_grad_(), b0.clone().requires_grad_()
    x2 = torch.linalg.solve(A2, b2)
    (0.5 * (x2 ** 2).sum() + x2[:, 1].sum()).backward()
    assert torch.allclose(x1, x2, rtol=1e-10, atol=1e-12)
    assert torch.allclose(A1.grad, A2.grad, rtol=1e-9, atol=1e-11)
    assert torch.allclose(b1.grad, b2.grad, rtol=1e-9, atol=1e-11)


def test_adjoint_many_rhs_odd_ld_and_errors(pkg):
    rng = np.random.default_rng(23)
    n, k = 333, 20
    A = rng.standard_normal((n, n)) + 3 * np.eye(n)
    F = pkg.lu(A)
    X = rng.standard_normal((n, k))
    Xb = rng.standard_normal((n, k))
    lam = np.linalg.solve(A.T, Xb)
    h = pkg.Handle.get()
    L = h.lib
    ldab = n + 1  # odd: the scalar store path
    Xc = torch.from_numpy(np.ascontiguousarray(X.T)).cuda()
    Xbc = torch.from_numpy(np.ascontiguousarray(Xb.T)).cuda()
    Bb = torch.empty_like(Xbc)
    Ab = torch.full((n, ldab), 7.0, dtype=torch.float64, device="cuda")
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    st = L.oxi_dlu_adjoint(h.ptr, n, k, vp(F._buf), F._lda, vp(F._ipiv), vp(Xc), n, vp(Xbc), n,
                           vp(Bb), n, vp(Ab), ldab)
    assert st == 0
    Abar = _np(Ab)[:, :n].T  # column j of Abar is row j of the buffer
    ref = -lam @ X.T
    assert np.abs(_np(Bb).T - lam).max() <= 1e-10 * np.abs(lam).max()
    assert np.abs(Abar - ref).max() <= 1e-10 * np.abs(ref).max()
    assert np.all(_np(Ab)[:, n] == 7.0)  # padding untouched
    # nrhs = 0: the gradient of A is zero
    st = L.oxi_dlu_adjoint(h.ptr, n, 0, vp(F._buf), F._lda, vp(F._ipiv), None, n, None, n, None, n,
                           vp(Ab), ldab)
    assert st == 0 and float(Ab[:, :n].abs().max()) == 0.0
    # Bbar aliasing Xbar with another leading dimension is rejected
    st = L.oxi_dlu_adjoint(h.ptr, n, k, vp(F._buf), F._lda, vp(F._ipiv), vp(Xc), n, vp(Xbc), n,
                           vp(Xbc), n + 1, vp(Ab), ldab)
    assert st == 1
    with pytest.raises(pkg.DimensionMismatch):
        pkg.lu_adjoint(F, torch.zeros(n + 1), torch.zeros(n + 1))


def _kappa_small(rng, n, kappa):
    U, R = np.linalg.qr(rng.standard_normal((n, n)))
    U *= np.sign(np.diag(R))
    V, R = np.linalg.qr(rng.standard_normal((n, n)))
    V *= np.sign(np.diag(R))
    s = 10.0 ** (-np.log10(kappa) * rng.uniform(0, 1, n))
    s[0], s[-1] = 1.0, 1.0 / kappa
    return (U * s) @ V.T


def test_batched_adjoint_1024_problems(pkg, oracle):
    """The batched rrule: 1024 problems, n ~ U{32..128}, kappa ~ 1e3 (the
    sigma-spectrum construction), loss 0.5||x||^2 per problem.  Each problem's
    (bbar, Abar) against the oracle's pullback from the same factors, and a
    sample against central finite differences (h = 1e-6)."""
    rng = np.random.default_rng(2026)
    orders = rng.integers(32, 129, 1024)
    mats = [_kappa_small(rng, int(n), 1e3) for n in orders]
    rhs = [rng.standard_normal(int(n)) for n in orders]
    P = pkg.BatchedLU(orders, np.ones_like(orders))
    P.load(mats, rhs)
    rep = P.gesv("fp64")
    assert np.all(rep["info"] == 0)
    xs = [_np(P.B(i))[:, 0].copy() for i in range(len(orders))]
    info = P.adjoint([x for x in xs])  # loss 0.5||x||^2: xbar = x
    assert np.all(info == 0)
    worst = 0.0
    for i in range(len(orders)):
        F, ip = _np(P.A(i)), _np(P.ipiv(i))
        bo, Ao = oracle.lu_adjoint(F, ip, xs[i], xs[i])
        bb, Ab = _np(P.Bbar(i))[:, 0], _np(P.Abar(i))
        worst = max(worst, np.linalg.norm(bb - bo) / np.linalg.norm(bo),
                    np.linalg.norm(Ab - Ao) / np.linalg.norm(Ao))
    # the two pullbacks associate the transposed solve's sums differently: they
    # agree to about kappa * n * eps (1e3 * 128 * 1.1e-16 = 1.4e-11)
    assert worst <= 1e-11, worst
    h = 1e-6
    for i in rng.choice(len(orders), 8, replace=False):
        A, b = mats[i], rhs[i]
        Ab = _np(P.Abar(i))
        bb = _np(P.Bbar(i))[:, 0]
        f = lambda M, v: 0.5 * np.sum(np.linalg.solve(M, v) ** 2)
        for _ in range(4):  # unit directions (Frobenius / 2-norm), as the single-matrix test
            dA = rng.standard_normal(A.shape)
            dA /= np.linalg.norm(dA)
            fd = (f(A + h * dA, b) - f(A - h * dA, b)) / (2 * h)
            assert abs(fd - np.sum(Ab * dA)) <= 1e-6 * max(1.0, abs(fd)), (i, fd)
            db = rng.standard_normal(b.shape)
            db /= np.linalg.norm(db)
            fd = (f(A, b + h * db) - f(A, b - h * db)) / (2 * h)
            assert abs(fd - bb @ db) <= 1e-6 * max(1.0, abs(fd)), (i, fd)


def test_batched_adjoint_several_rhs_and_edges(pkg, oracle):
    rng = np.random.default_rng(7)
    orders = np.array([1, 5, 64, 200, 256, 0])
    nrhs = np.array([1, 3, 8, 2, 4, 1])
    mats = [rng.standard_normal((n, n)) + n * np.eye(n) for n in orders]
    rhs = [rng.standard_normal((n, k)) for n, k in zip(orders, nrhs)]
    P = pkg.BatchedLU(orders, nrhs)
    P.load(mats, rhs)
    P.gesv("fp64")
    xbars = [rng.standard_normal((n, k)) for n, k in zip(orders, nrhs)]
    info = P.adjoint(xbars)
    assert np.all(info == 0)
    for i, n in enumerate(orders):
        if n == 0:
            continue
        X = _np(P.B(i))
        Ainv_T = np.linalg.inv(mats[i]).T
        bbar = Ainv_T @ xbars[i]
        assert np.allclose(_np(P.Bbar(i)), bbar, rtol=1e-11, atol=1e-13)
        assert np.allclose(_np(P.Abar(i)), -bbar @ X.T, rtol=1e-11, atol=1e-13)
    # a singular factor: the zero diagonal is reported
    S = rng.standard_normal((6, 6))
    S[:, 2] = 0.0
    Q = pkg.BatchedLU([6])
    Q.load([S], [rng.standard_normal(6)])
    Q.getrf()
    with pytest.raises(pkg.SingularException):
        Q.adjoint([np.ones(6)], solution="B")
