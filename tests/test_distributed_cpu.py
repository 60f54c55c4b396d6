"""The multi-GPU split of the batched path, checked on CPU with two gloo ranks.

Each rank takes its share of every size bucket (partition_by_bucket), computes
its problems' results -- here with the oracle on the host, standing in for the
GPU kernel -- and the final all-gather (gather_results) must give every rank
the results of the whole batch, equal to a single-process run.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import entry


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _batch(seed=5, count=300):
    rng = np.random.default_rng(seed)
    orders = rng.integers(1, 257, count)
    mats = []
    for i, n in enumerate(orders):
        A = rng.standard_normal((n, n)) + (n if i % 7 else 0) * np.eye(n)
        if i % 11 == 0 and n > 3:
            A[:, 2] = 0.0  # singular: info = 3
        mats.append(A)
    return orders, mats


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pkg = entry.load_package()
        from oxiblas_b200 import distributed as D
        orc = entry.load_oracle()
        orders, mats = _batch()
        idx = D.partition_by_bucket(orders, world)[rank]
        info = np.array([orc.getrf(mats[i], check=False)[2] for i in idx], dtype=np.int32)
        full = D.gather_results(len(orders), idx, {"info": info})
        np.save(out_path + f".{rank}.npy", full["info"])
    finally:
        dist.destroy_process_group()


def test_partition_covers_every_problem_once_and_balances():
    pkg = entry.load_package()
    from oxiblas_b200 import distributed as D
    rng = np.random.default_rng(1)
    orders = rng.integers(16, 257, 4096)
    for world in (1, 2, 3, 8):
        shards = D.partition_by_bucket(orders, world)
        allidx = np.concatenate(shards)
        assert np.array_equal(np.sort(allidx), np.arange(len(orders)))
        loads = [float(np.sum(orders[s].astype(float) ** 3)) for s in shards]
        assert max(loads) <= 1.02 * min(loads), (world, loads)
        # every bucket is spread over the ranks
        for b in range(8):
            members = np.nonzero((orders - 1) // 32 == b)[0]
            if len(members) >= 4 * world:
                per = [np.isin(s, members).sum() for s in shards]
                assert min(per) > 0, (world, b, per)
    a, b = D.partition_by_bucket(orders, 2), D.partition_by_bucket(orders, 2)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))  # deterministic


def test_gather_over_two_gloo_ranks_matches_one_process(tmp_path):
    orders, mats = _batch()
    orc = entry.load_oracle()
    serial = np.array([orc.getrf(A, check=False)[2] for A in mats], dtype=np.int32)
    assert np.any(serial > 0)
    out = str(tmp_path / "info")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    for r in range(2):
        got = np.load(out + f".{r}.npy")
        assert np.array_equal(got, serial), r
