#!/usr/bin/env python
"""Benchmark: n=16384 solve time, BF16-LU + FP64 iterative refinement vs plain
FP64 LU, at equal (FP64-level) backward error, on one B200 per rank.

One step = one solve of a seeded synthetic system A x = b with A = U diag(s) V^T
(Haar U, V; s log-uniform on [1e-4, 1], kappa ~ 1e4; n = 16384, one right-hand
side), factor + refinement until the normwise backward error
||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-14.  The matrix
(2.1 GB) is larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one system per rank, different seeds); the
LU of one matrix does not shard.  Rank 0 prints one JSON line.
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
    ap.add_argument("--prec", default="bf16x3", choices=["bf16x3", "bf16", "fp16", "fp32"])
    ap.add_argument("--refine", default="auto", choices=["ir", "gmres", "auto"])
    ap.add_argument("--tol", type=float, default=1e-14)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
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
# CPU oracle legs (baseline only; bounded samples extrapolated by flop count)
# ---------------------------------------------------------------------------
def lu_flops(n):
    return 2.0 / 3.0 * n ** 3


def prefix_flops(n, nb, steps):
    f = 0.0
    for s in range(steps):
        k = s * nb
        m = n - k
        # panel (m x nb), U block row TRSM, trailing update
        f += m * nb * nb + nb * nb * (n - k - nb) + 2.0 * (m - nb) * (n - k - nb) * nb
    return f


def cpu_mixed_estimate(A_np_colmajor_f32, n, panels=3):
    """FP32 LU prefix (first `panels` panels of 128 columns) on the host cores,
    extrapolated to the full factorization by flop count, plus one measured
    FP64 refinement iteration (FP64 residual + FP32 correction solve) times the
    iterations the reference's mixed_solve needs at this conditioning (3)."""
    import numpy as np
    import __graft_entry__ as E
    orc = E.load_oracle()
    W = A_np_colmajor_f32
    t0 = time.perf_counter()
    orc.getrf(W, blocksize=128, check=False, dtype=np.float32, steps=panels)
    t_prefix = time.perf_counter() - t0
    frac = prefix_flops(n, 128, panels) / lu_flops(n)
    t_lu = t_prefix / frac
    return t_lu, t_prefix, frac, orc.num_threads()


def cpu_refine_iteration(A64, x, b, LU32, ipiv):
    import numpy as np
    import __graft_entry__ as E
    orc = E.load_oracle()
    t0 = time.perf_counter()
    R, _ = orc.refinement_residual(A64, x, b)
    orc.getrs(LU32, ipiv, R.astype(np.float32))
    return time.perf_counter() - t0


def reference_arm(args, ws, rank):
    """The reference's own CPU implementation of the path, restated by the
    oracle (Julia is not installed): mixed_solve = FP32 LU + FP64 refinement,
    on all host cores, each step a bounded prefix sample extrapolated to the
    full n=16384 solve."""
    if rank != 0:
        return
    import numpy as np
    import __graft_entry__ as E
    orc = E.load_oracle()
    n = args.n
    rng = np.random.default_rng(20261104)
    A = np.asfortranarray(rng.standard_normal((n, n)).astype(np.float32))
    times = []
    for it in range(args.warmup + args.steps):
        W = A.copy(order="F")
        t_lu, t_prefix, frac, cores = cpu_mixed_estimate(W, n, panels=2)
        if it >= args.warmup:
            times.append(t_lu)
    # one refinement iteration at full size on a small factor stand-in: the
    # O(n^2) residual dominates it; the correction solve uses an identity factor
    x = np.zeros(n)
    b = rng.standard_normal(n)
    A64 = np.asfortranarray(A.astype(np.float64))
    t0 = time.perf_counter()
    orc.refinement_residual(A64, x, b)
    t_iter = time.perf_counter() - t0
    ms = (statistics.median(times) + 3 * t_iter) * 1e3
    cores = orc.num_threads()
    sample = (f"FP32 blocked LU (nb=128) of the first 2 panels of a 16384^2 matrix, extrapolated by "
              f"flop fraction {frac:.4f}, + 3 x one full-size FP64 residual ({t_iter*1e3:.0f} ms)")
    line = {"metric": METRIC, "value": round(ms, 3), "unit": "ms", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": n, "nrhs": 1},
            "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def ours(args, ws, rank, local):
    import numpy as np
    import torch
    import __graft_entry__ as E

    pkg = E.load_package()
    n = args.n
    dev = torch.device("cuda", local)
    seed = 20261104 + 7919 * rank
    A = pkg.synthetic.kappa_matrix(n, args.kappa, seed=seed, device=dev)
    g = torch.Generator(device=dev).manual_seed(seed + 1)
    b = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    Acm = A.t().contiguous()  # column-major A
    del A
    torch.cuda.empty_cache()
    Bcm = b.reshape(1, n).contiguous()
    Xcm = torch.zeros_like(Bcm)
    h = pkg.Handle.get()
    stream = torch.cuda.current_stream(dev)

    def mixed_step():
        st, rep = pkg.mixed_solve_device(Acm, Bcm, Xcm, n, 1, maxiter=30, rtol=args.tol,
                                         precision=args.prec, refine=args.refine, normwise=True)
        return st, rep

    # plain FP64 LU + solve through the C ABI (lu! on a copy, then ldiv!)
    work = torch.empty_like(Acm)
    xplain = torch.empty(n, dtype=torch.float64, device=dev)

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
    h.reset_launches()
    with Clocks(local) as ck:
        tot_mixed, per_mixed = timed(mixed_step, args.steps)
    launches = h.launches()
    clocks = ck.summary()
    st, rep = mixed_step()  # verification of the final state (untimed)
    ms_mixed = max_over_ranks(ws, tot_mixed / args.steps)

    # ---- timed: plain FP64 ----
    ksteps_plain = max(1, min(args.steps, 3))
    tot_plain, per_plain = timed(plain_step, ksteps_plain)
    ms_plain = max_over_ranks(ws, tot_plain / ksteps_plain)

    # backward errors of both answers (FP64, in the harness)
    def normwise(x):
        r = b - (Acm.t() @ x)
        an = Acm.t().abs().sum(dim=1).max()
        return float(r.abs().max() / (an * x.abs().max() + b.abs().max()))

    nw_mixed = normwise(Xcm[0])
    nw_plain = normwise(xplain)

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
    b_host = b.cpu().pin_memory()
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

    # ---- CPU baseline (rank 0, N=1) ----
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        A32 = np.asfortranarray(Acm.t().float().cpu().numpy())
        t_lu, t_prefix, frac, cores = cpu_mixed_estimate(A32, n, panels=3)
        del A32
        A64 = np.asfortranarray(Acm.t().cpu().numpy())
        x0 = Xcm[0].cpu().numpy()
        t0 = time.perf_counter()
        import __graft_entry__ as E2
        E2.load_oracle().refinement_residual(A64, x0, b.cpu().numpy())
        t_res = time.perf_counter() - t0
        del A64
        cpu_ms = (t_lu + 3 * t_res) * 1e3
        cpu = {"value": round(cpu_ms, 1), "unit": "ms", "cores": cores, "kind": "port",
               "sample": (f"oracle FP32 blocked LU (nb=128), first 3 panels of this 16384^2 matrix "
                          f"({t_prefix:.2f} s, flop fraction {frac:.4f}) extrapolated, + 3 x one "
                          f"full-size FP64 residual ({t_res*1e3:.0f} ms): the reference's mixed_solve")}

    line = {
        "metric": METRIC, "value": round(ms_mixed, 3), "unit": "ms", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_mixed, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": f"{args.prec}+f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "nrhs": 1, "kappa": args.kappa,
                   "precision": args.prec, "refine": args.refine, "stop": f"normwise<={args.tol}",
                   "l2": "inputs larger than L2 (2.1 GB matrix), no flush",
                   "parallelism": f"replicas{ws}"},
        "plain_fp64_ms": round(ms_plain, 3),
        "speedup_vs_plain_fp64": round(ms_plain / ms_mixed, 3),
        "backward_error_normwise": {"mixed": nw_mixed, "plain_fp64": nw_plain},
        "refinement": {"iterations": int(rep.iterations), "gmres_iterations": int(rep.gmres_iterations),
                       "refine_used": ("ir", "gmres", "auto")[rep.refine_used],
                       "factor_ms": round(rep.factor_ms, 3), "refine_ms": round(rep.refine_ms, 3)},
        "ms_per_step_each": [round(x, 3) for x in per_mixed],
        "roofline": roofline, "kernel_time_shares": shares,
        "plain_fp64_kernel_ms": plain_shares, "plain_fp64_trailing_gemm_tflops": plain_gemm_tflops,
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": n * n * 8 + n * 8,
                "d2h_bytes_per_step": n * 8},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, ws, rank)
        else:
            ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
