"""Seeded synthetic inputs with the shapes and value distributions of the
reference's benchmark and test configurations (no external datasets).

randn_shifted(n)      A = randn(n, n) + n*I  (benchmark/suite/inputs.jl:109-110)
kappa_matrix(n, k)    A = U diag(sigma) V^T, U and V Haar orthogonal (QR of a
                      seeded randn, signs fixed by diag(R)), sigma log-uniform on
                      [1/k, 1]: condition number ~k
"""
from __future__ import annotations

import torch


def _gen(seed: int, device):
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def randn_shifted(n: int, seed: int = 20261104, device="cuda", shift=None):
    g = _gen(seed, device)
    A = torch.randn(n, n, dtype=torch.float64, device=device, generator=g)
    A.diagonal().add_(float(n if shift is None else shift))
    return A


def haar_orthogonal(n: int, g, device="cuda"):
    Z = torch.randn(n, n, dtype=torch.float64, device=device, generator=g)
    Q, R = torch.linalg.qr(Z)
    Q *= torch.sign(torch.diagonal(R)).unsqueeze(0)
    return Q


def kappa_matrix(n: int, kappa: float, seed: int = 20261104, device="cuda",
                 row_scale_decades: float = 0.0):
    """U diag(sigma) V^T with sigma log-uniform on [1/kappa, 1]; optionally rows
    scaled by 10^U(-d, d) (the badly scaled large configuration)."""
    g = _gen(seed, device)
    U = haar_orthogonal(n, g, device)
    V = haar_orthogonal(n, g, device)
    lo = -torch.log10(torch.tensor(float(kappa), dtype=torch.float64))
    u = torch.rand(n, dtype=torch.float64, device=device, generator=g)
    sigma = 10.0 ** (lo.to(device) * u)
    sigma[0] = 1.0
    sigma[-1] = 1.0 / kappa
    A = (U * sigma.unsqueeze(0)) @ V.t()
    del U, V
    if row_scale_decades:
        d = float(row_scale_decades)
        rs = 10.0 ** ((torch.rand(n, dtype=torch.float64, device=device, generator=g) * 2 - 1) * d)
        A *= rs.unsqueeze(1)
    return A
