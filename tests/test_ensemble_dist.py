"""Ensemble sharding and the cross-rank FP64 reduction of S(k) (CPU, gloo, world size 2)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_members_once():
    from shhd_b200.ensemble import shard
    for members in (1, 7, 256, 257):
        for world in (1, 2, 3, 8):
            if world > members:
                continue
            seen = []
            for r in range(world):
                first, count = shard(members, world, r)
                seen.extend(range(first, first + count))
            assert seen == list(range(members))


def _worker(rank, world, port, members_per_rank, sk_per_rank, samples, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from shhd_b200.ensemble import reduce_structure_factor
        mean, total = reduce_structure_factor(np.array(sk_per_rank[rank]), samples, members_per_rank[rank])
        out[rank] = (mean.tolist(), total)
    finally:
        dist.destroy_process_group()


def test_reduce_structure_factor_two_ranks():
    rng = np.random.default_rng(3)
    samples = 5
    members = [3, 5]                                   # uneven shards
    # per-member S(k) samples; each rank's accumulator = sum over samples of its member mean
    per_member = [rng.random((samples, m, 4, 6)) for m in members]
    sk_rank = [pm.mean(axis=1).sum(axis=0) for pm in per_member]
    want = np.concatenate([pm for pm in per_member], axis=1).mean(axis=(0, 1))
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, members, [s.tolist() for s in sk_rank], samples, out))
                 for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        for r in range(2):
            mean, total = out[r]
            assert total == sum(members)
            assert np.allclose(np.array(mean), want, rtol=1e-14, atol=0)


def test_reduce_without_group_is_local_mean():
    from shhd_b200.ensemble import reduce_structure_factor
    acc = np.arange(12.0).reshape(3, 4)
    mean, total = reduce_structure_factor(acc, samples=4, members=2)
    assert total == 2
    assert np.allclose(mean, acc / 4)
