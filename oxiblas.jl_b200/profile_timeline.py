"""Launch timeline of one mixed-precision solve and one plain FP64 LU + solve.

Usage: python oxiblas.jl_b200/profile_timeline.py [--n 16384] [--nrhs 1] [--prec fp16x3] [--json out.json]
       python oxiblas.jl_b200/profile_timeline.py --kind cholesky [--n 8192]   (FP64 Cholesky, SPD G G^T + n I)
       python oxiblas.jl_b200/profile_timeline.py --kind complex [--n 4096]    (ComplexF64 LU of randn + i randn)

Runs the solves on the same seeded synthetic system as bench.py (Haar U, V,
sigma log-uniform on [1e-4, 1]) with the library's profiler on: every kernel
launch is bracketed by CUDA events on its own stream, so the timeline shows
which stream each kernel ran on (0: panels, 1: lookahead trailing update,
further: refinement) and when.  Profiled runs launch kernels one by one (no
graph replay), so their times are a little longer than bench.py's.
Prints a per-class and per-stream summary; --json writes the raw records
[(class, stream, start ms, end ms)].
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
from collections import defaultdict


def _load():
    here = os.path.dirname(os.path.abspath(__file__))
    if "oxiblas_b200" in sys.modules:
        return sys.modules["oxiblas_b200"]
    spec = importlib.util.spec_from_file_location("oxiblas_b200", os.path.join(here, "__init__.py"),
                                                  submodule_search_locations=[here])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["oxiblas_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def summarize(records, title):
    end = max(r[3] for r in records)
    print(f"== {title}: {len(records)} launches, span {end:.2f} ms")
    by = defaultdict(lambda: [0, 0.0])
    for r in records:
        by[r[0]][0] += 1
        by[r[0]][1] += r[3] - r[2]
    tot = sum(v[1] for v in by.values()) or 1.0
    for k, (c, ms) in sorted(by.items(), key=lambda kv: -kv[1][1]):
        print(f"  {k:10s} {c:6d} launches {ms:9.2f} ms  share {ms / tot:.3f}  mean {ms / c * 1e3:8.1f} us")
    for s in sorted({r[1] for r in records}):
        rs = [r for r in records if r[1] == s]
        busy = sum(r[3] - r[2] for r in rs)
        print(f"  stream {s}: {len(rs)} launches, busy {busy:.2f} ms, from {rs[0][2]:.2f} to {rs[-1][3]:.2f} ms")


def other_factorization(pkg, args):
    """Two warm-up factorizations, then one profiled: FP64 Cholesky of G G^T + n I
    or the ComplexF64 LU of a random complex matrix (seeded)."""
    import torch
    n = args.n
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(20261106)
    if args.kind == "cholesky":
        G = torch.randn(n, n, dtype=torch.float64, device=dev, generator=g)
        Acm = (G @ G.t() + n * torch.eye(n, dtype=torch.float64, device=dev)).t().contiguous()
        del G
        factor = pkg.cholesky_
    else:
        Acm = torch.complex(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g),
                            torch.randn(n, n, dtype=torch.float64, device=dev, generator=g)).t().contiguous()
        factor = pkg.lu_
    work = torch.empty_like(Acm)
    h = pkg.Handle.get()
    for _ in range(2):
        work.copy_(Acm)
        factor(work.t())
    torch.cuda.synchronize()
    work.copy_(Acm)
    h.profile(True)
    factor(work.t())
    tl = h.profile_timeline()
    h.profile(False)
    summarize(tl, f"{args.kind} factorization, n={n}")
    if args.json:
        with open(args.json, "w") as f:
            json.dump({args.kind: tl}, f)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--kappa", type=float, default=1e4)
    ap.add_argument("--prec", default="fp16x3")
    ap.add_argument("--json", default=None)
    ap.add_argument("--kind", default="lu", choices=["lu", "cholesky", "complex"])
    args = ap.parse_args()
    import torch
    pkg = _load()
    if args.kind != "lu":
        other_factorization(pkg, args)
        return
    n, nr = args.n, args.nrhs
    dev = torch.device("cuda", 0)
    A = pkg.synthetic.kappa_matrix(n, args.kappa, seed=20261104, device=dev)
    g = torch.Generator(device=dev).manual_seed(20261105)
    b = torch.randn(n, nr, dtype=torch.float64, device=dev, generator=g)
    Acm = A.t().contiguous()
    del A
    Bcm = b.t().contiguous()
    Xcm = torch.zeros_like(Bcm)
    h = pkg.Handle.get()

    def mixed():
        return pkg.mixed_solve_device(Acm, Bcm, Xcm, n, nr, maxiter=30, rtol=1e-14, precision=args.prec,
                                      refine="auto", normwise=True)

    work = torch.empty_like(Acm)
    x = torch.empty_like(b)

    def plain():
        work.copy_(Acm)
        F = pkg.lu_(work.t())
        x.copy_(b)
        F.ldiv_(x)

    for _ in range(2):
        mixed()
    plain()
    torch.cuda.synchronize()
    h.profile(True)
    mixed()
    tm = h.profile_timeline()
    h.profile(False)
    h.profile(True)
    plain()
    tp = h.profile_timeline()
    h.profile(False)
    summarize(tm, f"mixed {args.prec} solve, n={n}, nrhs={nr}")
    summarize(tp, f"plain FP64 LU + solve, n={n}, nrhs={nr}")
    if args.json:
        with open(args.json, "w") as f:
            json.dump({"mixed": tm, "plain": tp}, f)


if __name__ == "__main__":
    main()
