"""Ensemble sharding and the cross-rank FP64 reductions of S(k) and the Green-Kubo sums (CPU, gloo, world size 2)."""
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


# ---------------------------------------------------------------------------
# a real ensemble, computed by the oracle: sharded over two gloo ranks vs unsharded
# ---------------------------------------------------------------------------
ENSEMBLE_SCRIPT = """dimension 2
grid 16 16
length 16.0 16.0
dealias none
order_parameters 1
timestep 0.01
time_evolution srk3/incompressible
model free_energy quadratic a[0] 1.0
model transport constant eta 0.1 zeta 0.0 M[0,0] 0.5
fix 1 all nonlinear off
fix 2 all noise on seed 9 kBT 1.0
run 1
"""
MEMBERS, STEPS, NEVERY, NBLOCK, SK_EVERY = 5, 24, 2, 8, 6


def _oracle_member(m):
    """Member m's Green-Kubo sums and block count, and its S(k) of psi at every SK_EVERY-th step
    (oracle restatement of the engine's Philox noise, member key m)."""
    import shhd_oracle as so
    from helpers import random_state
    cfg = so.parse_script(ENSEMBLE_SCRIPT)
    u = random_state(cfg, seed=50 + m, amp=0.3, transverse=True)
    o = so.Oracle(cfg, member=m)
    gk = so.GreenKubo(cfg, NEVERY, NBLOCK)
    g = so.Geometry(cfg)
    sk = []
    for s in range(STEPS):
        u, flux = o.step_with_flux(u, "philox")
        gk.observe(flux)
        if (s + 1) % SK_EVERY == 0:
            sk.append(np.where(g.active, g.volume * np.abs(u[1]) ** 2 / g.grid_size ** 2, 0.0))
    return gk.sums, gk.nsample, np.array(sk)


def _shard_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from shhd_b200.ensemble import reduce_green_kubo, reduce_structure_factor, shard
        first, count = shard(MEMBERS, world, rank)
        res = [_oracle_member(m) for m in range(first, first + count)]
        gk_sums = sum(r[0] for r in res)
        gk_blocks = sum(r[1] for r in res)
        sk_acc = np.mean([r[2] for r in res], axis=0).sum(axis=0)   # sum over samples of the member mean
        s_mean, blocks = reduce_green_kubo(gk_sums, gk_blocks)
        sk_mean, members = reduce_structure_factor(sk_acc, STEPS // SK_EVERY, count)
        out[rank] = (s_mean.tolist(), blocks, sk_mean.tolist(), members)
    finally:
        dist.destroy_process_group()


def test_sharded_oracle_ensemble_matches_unsharded():
    """Green-Kubo S_mean and the structure factor of a 5-member ensemble stepped by the oracle,
    split 3 + 2 over two gloo ranks and reduced, equal the single-process ensemble values."""
    res = [_oracle_member(m) for m in range(MEMBERS)]
    want_s = sum(r[0] for r in res) / sum(r[1] for r in res)
    want_blocks = sum(r[1] for r in res)
    want_sk = np.mean([r[2] for r in res], axis=(0, 1))
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        for r in range(2):
            s_mean, blocks, sk_mean, members = out[r]
            assert blocks == want_blocks and members == MEMBERS
            assert np.allclose(np.array(s_mean), want_s, rtol=1e-13, atol=0)
            assert np.allclose(np.array(sk_mean), want_sk, rtol=1e-13, atol=1e-300)
