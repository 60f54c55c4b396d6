"""Mixed-precision solve on the GPU: the tcgen05 trailing-update kernel, the
reference properties of mixed_solve (test/lapack/factorizations.jl:57-63,
test/generic/extended_lapack.jl:97-117) and FP64-level backward error on
conditioned synthetic matrices."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("prec", ["bf16", "fp16", "bf16x3", "fp16x3", "fp32"])
def test_lowp_trailing_gemm(pkg, prec):
    torch.manual_seed(1)
    for (m, n, k) in ((128, 256, 64), (300, 517, 256), (2048, 1024, 256), (1000, 77, 40)):
        A = (torch.rand(m, k, device="cuda") * 2 - 1).float()  # |l| <= 1 like L21
        B = torch.randn(k, n, device="cuda").float() * 3
        C = torch.randn(m, n, device="cuda").float()
        C2 = C.clone()
        pkg.gemm_update_lowp(C2, A, B, prec)
        if prec == "bf16":  # exact products of BF16-rounded operands, FP32 accumulation
            ref = C.double() - A.bfloat16().double() @ B.bfloat16().double()
            tol = 1e-5
        else:  # scaled FP16, split BF16 and FP32 against the exact product
            ref = C.double() - A.double() @ B.double()
            tol = {"fp16": 5e-3, "bf16x3": 5e-5, "fp16x3": 1e-5, "fp32": 1e-5}[prec]
        err = (C2.double() - ref).abs().max().item() / ref.abs().max().item()
        assert err < tol, (prec, m, n, k, err)


@pytest.mark.parametrize("prec", ["fp32", "bf16", "fp16", "fp64", "bf16x3", "fp16x3"])
def test_mixed_solve_reference_cases(pkg, prec):
    rng = np.random.default_rng(7)
    for n in (1, 17, 67, 300):
        A = rng.standard_normal((n, n)) + n * np.eye(n)
        b = rng.standard_normal(n)
        r = pkg.mixed_solve(A, b, precision=prec)
        assert r["converged"] and r["iterations"] <= 10, (n, r)
        x = _np(r["x"])
        assert np.allclose(A @ x, b, rtol=2e-12, atol=2e-12)
        assert r["reason"] == "converged" and not r["fallback"]


def test_mixed_solve_options_and_errors(pkg):
    rng = np.random.default_rng(8)
    A = rng.standard_normal((40, 40)) + 40 * np.eye(40)
    b = rng.standard_normal(40)
    r = pkg.mixed_solve(A, b, maxiter=0, rtol=0.0)
    assert not r["converged"] and r["iterations"] == 0
    with pytest.raises(pkg.ArgumentError):
        pkg.mixed_solve(A, b, precision="int8")
    Ab = A.copy()
    Ab[3, 4] = np.nan
    with pytest.raises(pkg.ArgumentError):
        pkg.mixed_solve(Ab, b)
    B = rng.standard_normal((40, 5))
    r = pkg.mixed_solve(A, B, precision="bf16x3")
    assert r["converged"] and np.allclose(A @ _np(r["x"]), B, rtol=2e-12, atol=2e-12)


def test_mixed_low_precision_pivot_loss_falls_back(pkg):
    """1 + 2^-30 rounds to 1 in FP32: the low factor is exactly singular and the
    FP64 factor takes over (extended_lapack.jl:110-115, Float64 -> Float32)."""
    d = 2.0 ** -30
    A = np.array([[1.0, 1.0], [1.0, 1.0 + d]])
    b = np.array([2.0, 2.0 + d])
    r = pkg.mixed_solve(A, b, precision="fp32")
    assert r["fallback"] and r["reason"] == "working_factor_fallback" and r["converged"]
    assert np.allclose(_np(r["x"]), [1.0, 1.0], rtol=1e-10)
    with pytest.raises(pkg.SingularException):
        pkg.mixed_solve(A, b, precision="fp32", fallback=False)


@pytest.mark.parametrize("prec,refine,n,kappa", [("bf16x3", "ir", 1024, 1e4),
                                                 ("bf16x3", "auto", 1024, 1e4),
                                                 ("fp16x3", "ir", 1024, 1e4),
                                                 ("fp16x3", "auto", 2048, 1e4),
                                                 ("fp16", "gmres", 1024, 1e4),
                                                 ("fp32", "ir", 1024, 1e4),
                                                 ("bf16", "gmres", 512, 1e2)])
def test_mixed_conditioned_reaches_fp64_backward_error(pkg, oracle, prec, refine, n, kappa):
    """kappa 1e4: split BF16 converges with classical IR, FP16 needs GMRES-IR;
    single-pass BF16 (kappa * u_bf16 ~ 40 at 1e4) is exercised where GMRES-IR
    converges (kappa 1e2)."""
    A = pkg.synthetic.kappa_matrix(n, kappa, seed=11)
    g = torch.Generator(device="cuda").manual_seed(12)
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    r = pkg.mixed_solve(A, b, precision=prec, refine=refine, rtol=1e-14, normwise=True, maxiter=30)
    assert r["converged"], {k: v for k, v in r.items() if k != "x"}
    An, bn, x = _np(A), _np(b), _np(r["x"])
    assert oracle.normwise_backward_error(An, x, bn) <= 1e-14
    xo = np.linalg.solve(An, bn)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= kappa * 1e-13


@pytest.mark.parametrize("n", [129, 300, 1500, 4100])
def test_tournament_and_partial_pivoting_leaves_both_converge(pkg, oracle, n):
    """The mixed solve's FP32 factor with tournament-pivoting leaves (an option)
    and with the partial-pivoting leaves (default): both reach FP64 backward
    error, with similar iteration counts (the factor is a preconditioner for
    refinement)."""
    A = pkg.synthetic.kappa_matrix(n, 1e3, seed=21)
    g = torch.Generator(device="cuda").manual_seed(22)
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    its = {}
    for tour in (True, False):
        with pkg.options(tournament=tour):
            r = pkg.mixed_solve(A, b, precision="fp32", refine="ir", rtol=1e-14, normwise=True, maxiter=30)
        assert r["converged"], (tour, {k: v for k, v in r.items() if k != "x"})
        assert oracle.normwise_backward_error(_np(A), _np(r["x"]), _np(b)) <= 1e-14
        its[tour] = r["iterations"]
    assert its[True] <= its[False] + 2, its
    # a pivoting-hungry matrix (no diagonal dominance) through the 16-bit path
    rng = np.random.default_rng(23)
    An = rng.standard_normal((n, n))
    with pkg.options(tournament=True):
        r = pkg.mixed_solve(An, rng.standard_normal(n), precision="fp16x3", refine="auto", rtol=1e-14,
                            normwise=True, maxiter=30)
    assert r["converged"], {k: v for k, v in r.items() if k != "x"}


@pytest.mark.parametrize("prec", ["fp16x3", "fp32"])
def test_mixed_with_lookahead(pkg, oracle, prec):
    n = 2100
    A = pkg.synthetic.kappa_matrix(n, 1e4, seed=31)
    g = torch.Generator(device="cuda").manual_seed(32)
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    with pkg.options(lookahead=0):
        r0 = pkg.mixed_solve(A, b, precision=prec, refine="auto", rtol=1e-14, normwise=True, maxiter=30)
    with pkg.options(lookahead=1):
        r1 = pkg.mixed_solve(A, b, precision=prec, refine="auto", rtol=1e-14, normwise=True, maxiter=30)
        r2 = pkg.mixed_solve(A, b, precision=prec, refine="auto", rtol=1e-14, normwise=True, maxiter=30)
    for r in (r0, r1, r2):
        assert r["converged"]
        assert oracle.normwise_backward_error(_np(A), _np(r["x"]), _np(b)) <= 1e-14
    assert torch.equal(r1["x"], r2["x"])  # the graph replay of the lookahead schedule
    assert r1["iterations"] == r0["iterations"]
