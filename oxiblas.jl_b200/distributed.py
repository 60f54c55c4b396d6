"""Batched uneven LU across GPUs: one process per GPU, problems split by size
bucket, no collective on the data path.

The dense LU of one matrix does not shard (every panel depends on the one
before), so the multi-GPU form of the dense path is independent replicas.
The batched path does: its problems are independent.  Each rank takes a share
of every size bucket (orders 1..32, 33..64, ..., 225..256), assigned greedily
by cost (n^3, largest first, to the least loaded rank), factors and solves its
share with one BatchedLU launch on its own GPU, and a final all-gather brings
every problem's info, refinement steps and backward error to every rank -- the
only exchange, after the work.

The reference batches only its GEMM (gemm_batched!, src/blas/batched.jl:4-49:
an outer loop over independent problems split across threads); this is the
same split, across GPUs.
"""
from __future__ import annotations

import numpy as np

BUCKET = 32  # orders per size bucket (the batched kernel's buckets)


def partition_by_bucket(orders, world: int):
    """Indices of the problems each of `world` ranks takes: every size bucket
    is spread over all ranks, largest problems first, each to the rank with
    the least work so far (work = n^3).  Deterministic: every rank computes the
    same split from the same orders."""
    n = np.asarray(orders, dtype=np.int64).ravel()
    if world < 1:
        raise ValueError("world size must be positive")
    load = np.zeros(world, dtype=np.float64)
    shards = [[] for _ in range(world)]
    buckets = np.maximum(n - 1, 0) // BUCKET
    for b in np.unique(buckets)[::-1]:
        members = np.nonzero(buckets == b)[0]
        members = members[np.argsort(-n[members], kind="stable")]
        for i in members:
            r = int(np.argmin(load))
            shards[r].append(int(i))
            load[r] += float(n[i]) ** 3
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def gather_results(count: int, idx, fields: dict, group=None):
    """All-gather per-problem results (numpy arrays aligned with idx) into
    full arrays of `count` entries on every rank."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    mine = {"idx": np.asarray(idx, dtype=np.int64)}
    mine.update({k: np.asarray(v) for k, v in fields.items()})
    parts = [None] * world
    dist.all_gather_object(parts, mine, group=group)
    out = {}
    for k, v in fields.items():
        full = np.zeros(count, dtype=np.asarray(v).dtype)
        for p in parts:
            full[p["idx"]] = p[k]
        out[k] = full
    return out


def batched_gesv_sharded(As, Bs, prec: str = "fp64", maxiter: int = 10, rtol: float = 1e-13, group=None):
    """Factor and solve the batch with this rank's share on this process's GPU
    (torch.cuda.current_device()); returns (local indices, the local BatchedLU,
    gathered dict of info / iterations / backward_error for all problems)."""
    import torch.distributed as dist
    from .batched import BatchedLU
    orders = np.array([np.shape(a)[0] for a in As], dtype=np.int64)
    nrhs = np.array([np.reshape(b, (np.shape(b)[0], -1)).shape[1] for b in Bs], dtype=np.int64)
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    idx = partition_by_bucket(orders, world)[rank]
    P = BatchedLU(orders[idx], nrhs[idx]) if len(idx) else None
    fields = {"info": np.zeros(len(idx), np.int32), "iterations": np.zeros(len(idx), np.int32),
              "backward_error": np.zeros(len(idx), np.float64)}
    if P is not None:
        P.load([As[i] for i in idx], [Bs[i] for i in idx])
        rep = P.gesv(prec, maxiter=maxiter, rtol=rtol)
        fields["info"] = rep["info"]
        if prec == "fp32":
            fields["iterations"] = rep["iterations"]
            fields["backward_error"] = rep["backward_error"]
    full = gather_results(len(As), idx, fields, group) if world > 1 else fields
    return idx, P, full
