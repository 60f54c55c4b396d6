#!/usr/bin/env python
"""Benchmark: n=16384 solve time, 16-bit tensor-core LU + FP64 iterative
refinement vs plain FP64 LU, at equal (FP64-level) backward error, on one B200
per rank.  The default low precision is split FP16 (fp16x3: power-of-two
scaled FP16 operands, hi/lo split, three products per K on the tensor cores,
FP32 panels); split BF16 (bf16x3) is timed beside it on the same system.

One step = one solve of a seeded synthetic system A x = b with A = U diag(s) V^T
(Haar U, V; s log-uniform on [1e-4, 1], kappa ~ 1e4; n = 16384, one right-hand
side), factor + refinement until the normwise backward error
||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-14.  The matrix
(2.1 GB) is larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one system per rank, different seeds); the
LU of one matrix does not shard.  The batched workload splits one global batch
by size bucket over the ranks.  Without an external launcher (torchrun sets
WORLD_SIZE), --gpus N starts the N ranks itself.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "n=16384 solve time: BF16-LU+FP64 IR vs plain FP64 LU at equal backward error"
WORKLOAD = "dense LU solve n=16384 kappa~1e4 nrhs=1 (config 2 construction at the metric size)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--kappa", type=float, default=1e4)
    ap.add_argument("--prec", default="fp16x3", choices=["fp16x3", "bf16x3", "bf16", "fp16", "fp32"])
    ap.add_argument("--refine", default="auto", choices=["ir", "gmres", "auto"])
    ap.add_argument("--tol", type=float, default=1e-14)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--lookahead", type=int, default=None,
                    help="1: overlap each panel with the previous trailing update (both arms)")
    ap.add_argument("--workload", default="solve",
                    choices=["solve", "config2", "config5", "batched", "adjoint"],
                    help="solve: the headline n=16384 metric (default); config2: n=8192, 16 RHS, "
                         "kappa 1e4; config5: n=32768, kappa 1e6, rows scaled 10^U(-3,3), FP16 + "
                         "GMRES-IR; batched: 4096 uneven small LU solves in one launch; adjoint: rrule "
                         "of x = A \\ b at n=2048")
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--row-scale", type=float, default=0.0, help="rows scaled by 10^U(-d, d)")
    ap.add_argument("--alt", default="bf16x3", help="comma-separated precisions timed beside --prec")
    ap.add_argument("--count", type=int, default=4096, help="batched: number of problems")
    ap.add_argument("--no-autotune", action="store_true", help="batched: keep the default tuning")
    return ap.parse_args()


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region (clocks and throttle reasons)."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # nvidia-smi's start-up takes host CPU for a few hundred ms: let it
            # settle (first sample written) so it does not slow the timed steps'
            # host-side launches
            t0 = time.time()
            while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
            time.sleep(0.2)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path:
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = max(mx, float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU legs: the reference's own algorithm, restated by the oracle (Julia, the
# reference's language, is not installed), timed on the host cores
# ---------------------------------------------------------------------------
def lu_flops(n):
    return 2.0 / 3.0 * n ** 3


def load_synthetic():
    """The seeded input generator alone (torch only): the reference arm builds
    the GPU arm's system without importing the engine package."""
    import importlib.util
    path = os.path.join(ROOT, "oxiblas.jl_b200", "synthetic.py")
    spec = importlib.util.spec_from_file_location("oxiblas_synthetic", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def host_system(n, kappa, seed, nrhs, row_scale):
    """The GPU arm's seeded system (same generator, same seed) as host arrays:
    A column-major (Fortran order), B (n x nrhs)."""
    import numpy as np
    import torch
    syn = load_synthetic()
    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
    A = syn.kappa_matrix(n, kappa, seed=seed, device=dev, row_scale_decades=row_scale)
    g = torch.Generator(device=dev).manual_seed(seed + 1)
    b = torch.randn(n, nrhs, dtype=torch.float64, device=dev, generator=g)
    An = np.asfortranarray(A.cpu().numpy())
    bn = b.cpu().numpy()
    del A, b
    if torch.cuda.is_available():
        torch.cuda.empty_cache()
    return An, (bn[:, 0].copy() if nrhs == 1 else np.asfortranarray(bn))


def cpu_mixed_solve(orc, A, b, tol):
    """One full mixed_solve on the host cores: radix equilibration, FP32 LU
    (nb = 128, recursive panel, the reference's pivot rule and packed-GEMM
    order), FP64 residuals and corrections until the normwise backward error
    is <= tol (the GPU arm's stop test).  Returns (seconds, result dict)."""
    t0 = time.perf_counter()
    r = orc.mixed_solve_ex(A, b, maxiter=30, rtol=tol, normwise=True)
    return time.perf_counter() - t0, r


def reference_arm(args, ws, rank):
    """The reference's own CPU implementation of the path (mixed_solve, FP32 LU
    + FP64 refinement, src/lapack/extended_lapack.jl:175-226), restated by the
    oracle, on all host cores, on the GPU arm's system: every timed step is one
    full solve to the same stop test.  The warm-up steps solve a small system
    (threads and code warm; a full-size warm-up would add minutes)."""
    if rank != 0:
        return
    import numpy as np
    import __graft_entry__ as E
    orc = E.load_oracle()
    n = args.n
    A, b = host_system(n, args.kappa, 20261104, 1, args.row_scale)
    rng = np.random.default_rng(7)
    Aw = np.asfortranarray(rng.standard_normal((1024, 1024)) + 1024 * np.eye(1024))
    bw = rng.standard_normal(1024)
    for _ in range(args.warmup):
        cpu_mixed_solve(orc, Aw, bw, args.tol)
    times, res = [], None
    for _ in range(args.steps):
        dt, res = cpu_mixed_solve(orc, A, b, args.tol)
        times.append(dt)
    ms = statistics.mean(times) * 1e3
    cores = orc.num_threads()
    sample = (f"full run: every step one complete mixed_solve of the GPU arm's n={n} system "
              f"(seed 20261104): radix equilibration, FP32 blocked LU (nb=128), FP64 refinement to "
              f"normwise backward error <= {args.tol:g} ({res['iterations']} iterations, final "
              f"{res['backward_error_normwise']:.2e}); warm-up steps on a 1024^2 system")
    line = {"metric": METRIC, "value": round(ms, 3), "unit": "ms", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": n, "nrhs": 1, "kappa": args.kappa,
                       "stop": f"normwise<={args.tol}"},
            "refinement": {"iterations": res["iterations"],
                           "backward_error_normwise": res["backward_error_normwise"],
                           "backward_error": res["backward_error"], "converged": res["converged"]},
            "ms_per_step_each": [round(t * 1e3, 1) for t in times],
            "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def ours(args, ws, rank, local, metric=METRIC, workload=WORKLOAD):
    import numpy as np
    import torch
    import __graft_entry__ as E

    pkg = E.load_package()
    n = args.n
    dev = torch.device("cuda", local)
    seed = 20261104 + 7919 * rank
    nrhs = args.nrhs
    A = pkg.synthetic.kappa_matrix(n, args.kappa, seed=seed, device=dev, row_scale_decades=args.row_scale)
    g = torch.Generator(device=dev).manual_seed(seed + 1)
    b = torch.randn(n, nrhs, dtype=torch.float64, device=dev, generator=g)
    Acm = A.t().contiguous()  # column-major A
    del A
    torch.cuda.empty_cache()
    Bcm = b.t().contiguous()  # (nrhs, n): column-major B
    Xcm = torch.zeros_like(Bcm)
    h = pkg.Handle.get()
    if args.lookahead is not None:
        h.set_option(4, args.lookahead)  # OXI_OPT_LOOKAHEAD, for the mixed and the plain arm
    stream = torch.cuda.current_stream(dev)

    def mixed_step():
        st, rep = pkg.mixed_solve_device(Acm, Bcm, Xcm, n, nrhs, maxiter=30, rtol=args.tol,
                                         precision=args.prec, refine=args.refine, normwise=True)
        return st, rep

    # plain FP64 LU + solve through the C ABI (lu! on a copy, then ldiv!)
    work = torch.empty_like(Acm)
    xplain = torch.empty(n, nrhs, dtype=torch.float64, device=dev)

    def plain_step():
        work.copy_(Acm)
        F = pkg.lu_(work.t())
        xplain.copy_(b)
        F.ldiv_(xplain)
        return F

    def timed(fn, steps):
        barrier(ws)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        per = []
        e0.record(stream)
        for _ in range(steps):
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            fn()
            s1.record(stream)
            per.append((s0, s1))
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        tot = e0.elapsed_time(e1)
        return tot, [a.elapsed_time(bb) for a, bb in per]

    # ---- warm-up ----
    for _ in range(args.warmup):
        st, rep = mixed_step()
    assert rep.converged, f"mixed solve did not converge (status {st})"
    for _ in range(max(1, min(args.warmup, 2))):
        plain_step()

    # ---- timed: mixed (value) ----
    with Clocks(local) as ck:
        for _ in range(2):  # the GPU idled while the sampler started: bring its clocks back up
            mixed_step()
        h.reset_launches()
        tot_mixed, per_mixed = timed(mixed_step, args.steps)
    launches = h.launches()
    clocks = ck.summary()
    st, rep = mixed_step()  # verification of the final state (untimed)
    ms_mixed = max_over_ranks(ws, tot_mixed / args.steps)

    # ---- other low precisions on the same system, for comparison ----
    alt = {}
    for ap_ in [a for a in args.alt.split(",") if a and a != args.prec]:
        def alt_step(prec=ap_):
            return pkg.mixed_solve_device(Acm, Bcm, Xcm, n, nrhs, maxiter=30, rtol=args.tol, precision=prec,
                                          refine=args.refine, normwise=True)
        for _ in range(2):
            alt_step()
        ka = max(1, min(args.steps, 3))
        tot_a, _ = timed(alt_step, ka)
        st_a, rep_a = alt_step()
        alt[ap_] = {"ms": round(max_over_ranks(ws, tot_a / ka), 3), "iterations": int(rep_a.iterations),
                    "gmres_iterations": int(rep_a.gmres_iterations), "converged": bool(rep_a.converged)}
    if alt:
        mixed_step()  # leave the default precision's answer in Xcm

    # ---- timed: plain FP64 ----
    ksteps_plain = max(1, min(args.steps, 3))
    tot_plain, per_plain = timed(plain_step, ksteps_plain)
    ms_plain = max_over_ranks(ws, tot_plain / ksteps_plain)

    # backward errors of both answers (FP64, in the harness)
    def normwise(x):  # max over right-hand sides of ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)
        r = b - (Acm.t() @ x)
        an = Acm.t().abs().sum(dim=1).max()
        return float((r.abs().amax(dim=0) / (an * x.abs().amax(dim=0) + b.abs().amax(dim=0))).max())

    nw_mixed = normwise(Xcm.t())
    nw_plain = normwise(xplain)
    fwd_vs_plain = float((Xcm.t() - xplain).abs().max() / xplain.abs().max())

    # ---- profiled pass (same steps) for the roofline of the dominant kernel ----
    h.profile(True)
    torch.cuda.synchronize()
    for _ in range(args.steps):
        mixed_step()
    prof = h.profile_read()
    h.profile(False)
    peaks, peak_kind = load_peaks()
    total_ms = sum(v[1] for v in prof.values()) or 1.0
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    roofline = None
    if dom:
        name, (cnt, ms, fl, by) = dom
        hbm = peaks.get("hbm_gbs", 6650.0)
        achieved = by / (ms / 1e3) / 1e9
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic_per_launch.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                traffic = json.load(f).get(name)
        roofline = {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1),
                    "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                    "traffic": traffic, "peak_source": peak_kind,
                    "launches": cnt, "avg_launch_us": round(ms / cnt * 1e3, 2),
                    "algorithmic_bytes_per_launch": round(by / cnt),
                    "algorithmic_flops_per_launch": round(fl / cnt)}
        if fl / max(by, 1) > peaks.get("bf16_tflops", 1590.0) * 1e3 / hbm:
            tf = fl / (ms / 1e3) / 1e12
            roofline.update({"bound": "tensor", "achieved": round(tf, 2),
                             "peak": peaks.get("bf16_tflops"), "unit": "TFLOP/s",
                             "frac": round(tf / peaks.get("bf16_tflops"), 4)})
    shares = {k: round(v[1] / total_ms, 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])}
    # kernel-class breakdown of one plain FP64 step (diagnostic)
    h.profile(True)
    plain_step()
    pprof = h.profile_read()
    h.profile(False)
    ptot = sum(v[1] for v in pprof.values()) or 1.0
    plain_shares = {k: [round(v[1], 3), v[0]] for k, v in sorted(pprof.items(), key=lambda kv: -kv[1][1])}
    dmma = pprof.get("gemm_dmma")
    plain_gemm_tflops = round(dmma[2] / (dmma[1] / 1e3) / 1e12, 2) if dmma else None

    # ---- e2e through the public API (host buffers, copies inside the region) ----
    A_host = Acm.t().cpu().pin_memory()  # the user's row-indexed matrix on the host
    b_host = (b[:, 0] if nrhs == 1 else b).cpu().pin_memory()
    ke = max(1, min(args.steps, 3))
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(ke):
        r = pkg.mixed_solve(A_host, b_host, maxiter=30, rtol=args.tol, precision=args.prec,
                            refine=args.refine, normwise=True)
        x_host = r["x"].cpu()
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(ws, ev0.elapsed_time(ev1) / ke)
    assert r["converged"]
    del A_host

    # ---- CPU baseline (rank 0, N=1): one full solve of this system ----
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu and metric == METRIC:
        orc = E.load_oracle()
        A64 = np.asfortranarray(Acm.t().cpu().numpy())
        b64 = b[:, 0].cpu().numpy()
        t_cpu, rc = cpu_mixed_solve(orc, A64, b64, args.tol)
        del A64
        cpu = {"value": round(t_cpu * 1e3, 1), "unit": "ms", "cores": orc.num_threads(), "kind": "port",
               "sample": (f"full run: one complete mixed_solve of this n={n} system on the host cores "
                          f"(oracle restatement: radix equilibration, FP32 blocked LU nb=128, FP64 "
                          f"refinement to normwise <= {args.tol:g}: {rc['iterations']} iterations, "
                          f"final {rc['backward_error_normwise']:.2e})")}

    line = {
        "metric": metric, "value": round(ms_mixed, 3), "unit": "ms", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_mixed, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": f"{args.prec}+f32+f64", "data": "synthetic",
        "config": {"workload": workload, "n": n, "nrhs": nrhs, "kappa": args.kappa,
                   "row_scale_decades": args.row_scale,
                   "precision": args.prec, "refine": args.refine, "stop": f"normwise<={args.tol}",
                   "l2": "inputs larger than L2 (2.1 GB matrix), no flush",
                   "lookahead": int(args.lookahead or 0), "parallelism": f"replicas{ws}"},
        "plain_fp64_ms": round(ms_plain, 3),
        "speedup_vs_plain_fp64": round(ms_plain / ms_mixed, 3),
        "backward_error_normwise": {"mixed": nw_mixed, "plain_fp64": nw_plain},
        "forward_error_vs_plain_fp64": fwd_vs_plain,
        "refinement": {"iterations": int(rep.iterations), "gmres_iterations": int(rep.gmres_iterations),
                       "refine_used": ("ir", "gmres", "auto")[rep.refine_used],
                       "factor_ms": round(rep.factor_ms, 3), "refine_ms": round(rep.refine_ms, 3)},
        "ms_per_step_each": [round(x, 3) for x in per_mixed],
        "other_precisions": alt,
        "roofline": roofline, "kernel_time_shares": shares,
        "plain_fp64_kernel_ms": plain_shares, "plain_fp64_trailing_gemm_tflops": plain_gemm_tflops,
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": n * n * 8 + n * nrhs * 8,
                "d2h_bytes_per_step": n * nrhs * 8},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Secondary workloads (not the headline line): batched uneven LU, adjoint
# ---------------------------------------------------------------------------
def _timed_each(stream, fn, steps, pre=None):
    import torch
    out = []
    for _ in range(steps):
        if pre:
            pre()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def batched_workload(args, ws, rank, local):
    """4096 independent FP64 systems, n ~ U{16..256}, A = N(0,1) + n I, 1..8 RHS:
    FP32 factor + FP64 refinement (componentwise 1e-13) vs plain FP64, each one
    persistent launch over all problems."""
    import numpy as np
    import torch
    import __graft_entry__ as E
    pkg = E.load_package()
    dev = torch.device("cuda", local)
    # one global batch (the same seed on every rank); with N ranks each takes
    # its share of every size bucket (no collective until the timing's max)
    rng = np.random.default_rng(20261104)
    count_all = args.count
    orders_all = rng.integers(16, 257, size=count_all)
    k_all = rng.integers(1, 9, size=count_all)
    from oxiblas_b200 import distributed as D
    mine = D.partition_by_bucket(orders_all, ws)[rank]
    orders, k = orders_all[mine], k_all[mine]
    count = len(orders)
    P = pkg.BatchedLU(orders, k, device=dev)
    g = torch.Generator(device=dev).manual_seed(20261104 + rank)
    P.poolA.normal_(generator=g)
    P.poolB.normal_(generator=g)
    diag = np.concatenate([P._offA[i] + np.arange(n) * (n + 1) for i, n in enumerate(orders)])
    dshift = np.concatenate([np.full(n, float(n)) for n in orders])
    P.poolA[torch.from_numpy(diag).to(dev)] += torch.from_numpy(dshift).to(dev)
    A0, B0 = P.poolA.clone(), P.poolB.clone()
    tune = None
    if not args.no_autotune:
        tune = {"fp32": pkg.batched_autotune(orders, "fp32", nrhs=4)[:2],
                "fp64": pkg.batched_autotune(orders, "fp64", nrhs=4)[:2]}
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        rep = P.gesv("fp32", maxiter=10, rtol=1e-13)
    h = pkg.Handle.get()
    with Clocks(local) as ck:
        for _ in range(2):  # the GPU idled while the sampler started: bring its clocks back up
            P.gesv("fp32", maxiter=10, rtol=1e-13)
        h.reset_launches()
        t_mixed = _timed_each(stream, lambda: P.gesv("fp32", maxiter=10, rtol=1e-13), args.steps)
    launches = h.launches() // max(1, args.steps)
    clocks = ck.summary()
    rep = P.gesv("fp32", maxiter=10, rtol=1e-13)

    def restore():
        P.poolA.copy_(A0)
        P.poolB.copy_(B0)

    for _ in range(max(1, args.warmup)):
        restore()
        P.gesv("fp64")
    t_plain = _timed_each(stream, lambda: P.gesv("fp64"), args.steps, pre=restore)
    ms_mixed = max_over_ranks(ws, statistics.median(t_mixed))
    ms_plain = max_over_ranks(ws, statistics.median(t_plain))
    flops = float(np.sum(2.0 / 3.0 * orders_all.astype(float) ** 3 + 2.0 * orders_all.astype(float) ** 2 * k_all))
    # plain FP64: read A, write LU, read B, write X once (algorithmic bytes)
    bytes_plain = float(np.sum(16.0 * orders_all.astype(float) ** 2 + 16.0 * orders_all * k_all))
    # check a sample of the plain answers against the untouched copy
    restore()
    Bref = B0.clone()
    P.gesv("fp64")
    worst = 0.0
    for i in range(0, count, max(1, count // 64)):
        n, kk = int(orders[i]), int(k[i])
        Ai = A0[P._offA[i]:P._offA[i] + n * n].view(n, n).t()
        Bi = Bref[P._offB[i]:P._offB[i] + n * kk].view(kk, n).t()
        Xi = P.B(i)
        R = Bi - Ai @ Xi
        den = Ai.abs() @ Xi.abs() + Bi.abs()
        worst = max(worst, float((R.abs() / den).max()))
    line = {
        "metric": "batched uneven LU+solve time: 4096 FP64 systems, n~U{16..256}, 1-8 RHS",
        "value": round(ms_mixed, 3), "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_mixed, 3), "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"batched uneven LU, {count_all} problems, n~U{{16..256}}, N(0,1)+nI, "
                               "nrhs~U{1..8}; one persistent graph-replayed launch per GPU",
                   "l2": "pools (≈0.8 GB) larger than L2",
                   "parallelism": f"problems split by size bucket over {ws} GPU(s)"},
        "plain_fp64_ms": round(ms_plain, 3),
        "speedup_vs_plain_fp64": round(ms_plain / ms_mixed, 3),
        "tflops": {"mixed": round(flops / ms_mixed / 1e9, 3), "plain_fp64": round(flops / ms_plain / 1e9, 3)},
        "plain_fp64_hbm_gbs": round(bytes_plain / ms_plain / 1e6, 1),
        "refinement": {"max_iterations": int(rep["iterations"].max()),
                       "mean_iterations": round(float(rep["iterations"].mean()), 3),
                       "max_backward_error": float(rep["backward_error"].max())},
        "plain_fp64_max_backward_error_sample": worst,
        "tuning": tune, "gpu_launches_per_step": launches, "clocks": clocks,
        "ms_each": {"mixed": [round(x, 3) for x in t_mixed], "plain_fp64": [round(x, 3) for x in t_plain]},
    }
    if not args.no_cpu and rank == 0 and ws == 1:
        orc = E.load_oracle()
        sample = list(range(0, count, 16))
        An = A0.cpu().numpy()
        Bn = B0.cpu().numpy()
        t0 = time.perf_counter()
        for i in sample:
            n, kk = int(orders[i]), int(k[i])
            Ai = An[P._offA[i]:P._offA[i] + n * n].reshape(n, n).T
            Bi = Bn[P._offB[i]:P._offB[i] + n * kk].reshape(kk, n).T
            F, ip, _ = orc.getrf(Ai, check=False)
            orc.getrs(F, ip, Bi)
        t_s = time.perf_counter() - t0
        fs = float(np.sum(2.0 / 3.0 * orders[sample].astype(float) ** 3))
        ft = float(np.sum(2.0 / 3.0 * orders.astype(float) ** 3))
        line["cpu_baseline"] = {"value": round(t_s * ft / fs * 1e3, 1), "unit": "ms", "cores": orc.num_threads(),
                                "kind": "port",
                                "sample": f"oracle FP64 getrf+getrs on every 16th problem ({len(sample)}), "
                                          "extrapolated by LU flops"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def adjoint_workload(args, ws, rank, local):
    """rrule of x = A \\ b, n = 2048, kappa 1e3: pullback time with the stored factors; the
    batched rrule (1024 problems, n ~ U{32..128}) beside it."""
    import torch
    import __graft_entry__ as E
    pkg = E.load_package()
    dev = torch.device("cuda", local)
    n = 2048
    A = pkg.synthetic.kappa_matrix(n, 1e3, seed=4242 + rank, device=dev)
    g = torch.Generator(device=dev).manual_seed(4243 + rank)
    b = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    F = pkg.lu(A)
    x = F.solve(b)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        pkg.lu_adjoint(F, x, x)
    t = _timed_each(stream, lambda: pkg.lu_adjoint(F, x, x), args.steps)

    def fwd_bwd():
        A1 = A.clone().requires_grad_()
        xx = pkg.solve(A1, b)
        (0.5 * (xx * xx).sum()).backward()

    for _ in range(args.warmup):
        fwd_bwd()
    t2 = _timed_each(stream, fwd_bwd, args.steps)

    # the batched rrule: 1024 problems, n ~ U{32..128}, N(0,1) + n I, one
    # right-hand side each, loss 0.5||x||^2 (xbar = x): the batched FP64 solve,
    # then the pullback of every problem from the stored factors
    import numpy as np
    rng = np.random.default_rng(20261105)
    orders = rng.integers(32, 129, size=1024)
    P = pkg.BatchedLU(orders, np.ones_like(orders), device=dev)
    gb = torch.Generator(device=dev).manual_seed(4244 + rank)
    P.poolA.normal_(generator=gb)
    P.poolB.normal_(generator=gb)
    diag = np.concatenate([P._offA[i] + np.arange(m) * (m + 1) for i, m in enumerate(orders)])
    P.poolA[torch.from_numpy(diag).to(dev)] += torch.from_numpy(
        np.concatenate([np.full(m, float(m)) for m in orders])).to(dev)
    A0, B0 = P.poolA.clone(), P.poolB.clone()

    def restore():
        P.poolA.copy_(A0)
        P.poolB.copy_(B0)

    for _ in range(args.warmup):
        restore()
        P.gesv("fp64")
    tb_fwd = _timed_each(stream, lambda: P.gesv("fp64"), args.steps, pre=restore)
    P._adjoint_pools()
    P.poolXbar.copy_(P.poolB)
    for _ in range(args.warmup):
        P.adjoint()
    tb_bwd = _timed_each(stream, lambda: P.adjoint(), args.steps)
    ms = max_over_ranks(ws, statistics.median(t))
    line = {"metric": "adjoint of x = A\\b (n=2048, kappa 1e3): pullback time with stored LU factors",
            "value": round(ms, 4), "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "rrule x = A\\b, n=2048, sigma log-uniform [1e-3, 1], loss 0.5||x||^2",
                       "parallelism": f"replicas{ws}"},
            "forward_plus_backward_ms": round(max_over_ranks(ws, statistics.median(t2)), 4),
            "abar_write_gbs": round(8.0 * n * n / (ms / 1e3) / 1e9, 1),
            "batched_1024": {"workload": "1024 problems, n~U{32..128}, N(0,1)+nI, 1 RHS, loss 0.5||x||^2",
                             "forward_solve_ms": round(max_over_ranks(ws, statistics.median(tb_fwd)), 4),
                             "pullback_ms": round(max_over_ranks(ws, statistics.median(tb_bwd)), 4)}}
    if rank == 0:
        print(json.dumps(line), flush=True)


def _spawned_rank(rank, world, port, argv):
    """One rank of a self-launched multi-GPU run (no external launcher)."""
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.argv = argv
    main()


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # `bench.py --gpus N` on its own: start the N ranks here, one process per
        # GPU (torchrun sets WORLD_SIZE and comes straight through)
        import socket
        import torch.multiprocessing as mp
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        mp.spawn(_spawned_rank, args=(args.gpus, port, list(sys.argv)), nprocs=args.gpus, join=True)
        return
    ws, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, ws, rank)
        elif args.workload == "batched":
            batched_workload(args, ws, rank, local)
        elif args.workload == "adjoint":
            adjoint_workload(args, ws, rank, local)
        elif args.workload == "config2":
            args.n, args.nrhs, args.kappa = 8192, 16, 1e4
            ours(args, ws, rank, local,
                 metric="n=8192 16-RHS solve time: 16-bit tensor-core LU + FP64 IR vs plain FP64 LU "
                        "at equal backward error (kappa 1e4)",
                 workload="dense LU solve n=8192 kappa~1e4 nrhs=16 (Haar U, V; sigma log-uniform)")
        elif args.workload == "config5":
            args.n, args.nrhs, args.kappa, args.row_scale = 32768, 1, 1e6, 3.0
            if args.alt == "bf16x3":  # single-pass FP16 + GMRES-IR (the configuration's form) beside it
                args.alt = "fp16"
            ours(args, ws, rank, local,
                 metric="n=32768 solve time, kappa 1e6 and rows scaled 10^U(-3,3): FP16 tensor-core LU + "
                        "FP64 GMRES-IR vs plain FP64 LU at equal backward error",
                 workload="dense LU solve n=32768 kappa~1e6, row scaling 10^U(-3,3), nrhs=1")
        else:
            ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
