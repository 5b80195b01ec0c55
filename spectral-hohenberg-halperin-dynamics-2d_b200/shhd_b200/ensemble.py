"""Ensembles sharded over ranks (one process per GPU).

Members are independent, so a many-member ensemble shards across ranks with
no exchange during the run: rank r advances members [r * M, (r + 1) * M) of
the ensemble (their noise keys are member_offset + m, so the union over ranks
is the same ensemble whatever the rank count).  The collectives are sums
of the FP64 measure accumulators at read-out: each rank holds the sum of its
members' S(k) samples (a per-rank mean over its members, times the number of
samples), and the ensemble mean is the member-weighted mean over ranks; the
Yokota-Green-Kubo sums and block counts of every member add up the same way.
(The reference's own MPI_Reduce of the Green-Kubo integrals,
measure_yokota_green_kubo.cc:166, sums one trajectory's partial Fourier sums
over its x-slabs; here a trajectory lives on one GPU and the ranks hold
different realisations, so what crosses ranks is the finished FP64 sums.)
"""
from __future__ import annotations

from typing import Tuple

import numpy as np


def shard(members: int, world: int, rank: int) -> Tuple[int, int]:
    """(first member, member count) of `rank` when `members` are split over `world` ranks."""
    if members < 1 or world < 1 or not 0 <= rank < world:
        raise ValueError("need members >= 1 and 0 <= rank < world")
    base, extra = divmod(members, world)
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def reduce_structure_factor(sk_sum: np.ndarray, samples: int, members: int, group=None, device=None) -> Tuple[np.ndarray, int]:
    """Ensemble-mean S(k) over all ranks.

    `sk_sum` is this rank's accumulator (sum over `samples` samples of the mean
    over its `members` members, as `Engine.sk_read` returns it).  Every rank
    must take the same number of samples.  Returns (mean S(k) over all members
    and samples, total members).  One all-reduce (FP64) of the member-weighted
    sums; without an initialised process group the local mean is returned.
    """
    import torch
    import torch.distributed as dist

    if samples < 1:
        raise ValueError("no samples")
    weighted = np.ascontiguousarray(sk_sum, dtype=np.float64) * float(members)
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return weighted / (members * samples), members
    t = torch.from_numpy(np.concatenate([weighted.ravel(), [float(members), float(samples)]]))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = t.cpu().numpy()
    total_members = out[-2]
    total_samples = out[-1] / dist.get_world_size(group)
    if abs(total_samples - samples) > 1e-9:
        raise RuntimeError("ranks took different numbers of samples")
    return out[:-2].reshape(np.shape(sk_sum)) / (total_members * samples), int(round(total_members))


def reduce_green_kubo(sums: np.ndarray, blocks: int, group=None, device=None) -> Tuple[np.ndarray, int]:
    """Ensemble Yokota-Green-Kubo estimate over all ranks.

    `sums` is this rank's [tau, mode] sum over its members of Engine.gk_read's sums (each the
    sum over that member's completed blocks of |I|^2 / (2 tau kBT V)), `blocks` the total of
    their completed blocks.  Returns (S_mean = all sums / all blocks, as the reference's
    sum / nsample over every block of every member, and the total block count): one FP64
    all-reduce of the sums with the count appended; without a process group the local values.
    """
    import torch
    import torch.distributed as dist

    local = np.ascontiguousarray(sums, dtype=np.float64)
    if group is None and not (dist.is_available() and dist.is_initialized()):
        total = float(blocks)
        out = local
    else:
        t = torch.from_numpy(np.concatenate([local.ravel(), [float(blocks)]]))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        arr = t.cpu().numpy()
        total = arr[-1]
        out = arr[:-1].reshape(local.shape)
    if total < 1:
        raise ValueError("no completed Green-Kubo blocks on any rank")
    return out / total, int(round(total))
