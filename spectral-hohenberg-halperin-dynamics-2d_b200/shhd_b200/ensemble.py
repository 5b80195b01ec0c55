"""Ensembles sharded over ranks (one process per GPU).

Members are independent, so a many-member ensemble shards across ranks with
no exchange during the run: rank r advances members [r * M, (r + 1) * M) of
the ensemble (their noise keys are member_offset + m, so the union over ranks
is the same ensemble whatever the rank count).  The one collective is the sum
of the FP64 measure accumulators at read-out: each rank holds the sum of its
members' S(k) samples (a per-rank mean over its members, times the number of
samples), and the ensemble mean is the member-weighted mean over ranks.
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
