"""Multi-process host logic of the replicas / sharded path, on CPU with gloo
(world size 2): cost-balanced sharding covers every instance once, and the result
gather restores input order.  The per-rank evaluation here is the oracle (CPU);
on GPUs it is the single-GPU queue."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gbskernels_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, funcs, mats, q):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = D.shard(funcs, [m.shape[0] for m in mats], world)
        mine = parts[rank]
        vals = [getattr(oracle, funcs[i])(mats[i]) for i in mine]
        out = D.gather_results(mine, vals, len(mats))
        q.put((rank, parts, out))
    finally:
        dist.destroy_process_group()


def test_shard_is_a_balanced_partition():
    rng = np.random.default_rng(0)
    funcs = list(rng.choice(["haf", "lhaf", "tor", "perm"], size=200))
    dims = [int(rng.integers(2, 12)) * 2 for _ in range(200)]
    for world in (1, 2, 3, 8):
        parts = D.shard(funcs, dims, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(200))
        loads = [sum(D.instance_cost(funcs[i], dims[i]) for i in p) for p in parts]
        assert max(loads) <= sum(loads) / world + max(D.instance_cost(f, d) for f, d in zip(funcs, dims))


def test_two_rank_gloo_gather_restores_order(orc):
    rng = np.random.default_rng(1)
    funcs, mats = [], []
    for k in range(12):
        N = int(rng.integers(1, 5)) * 2
        X = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        funcs.append(["haf", "lhaf"][k % 2])
        mats.append((X + X.T) / 2)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, funcs, mats, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import oracle
    expect = np.array([getattr(oracle, f)(m) for f, m in zip(funcs, mats)])
    for rank, parts, out in res:
        assert sorted(parts[0] + parts[1]) == list(range(12))
        assert np.array_equal(out, expect)
