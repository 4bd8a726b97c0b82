"""History sharding over ranks and the one tally exchange.

Histories are independent: rank r of W simulates its own contiguous range
of history indices (disjoint Philox counters, so no two ranks share a
stream) and keeps a private FP64 grid.  The single exchange step is a sum of
the tally arrays, the statistics arrays and the counters over ranks, done
with torch.distributed (NCCL on GPUs, gloo on CPUs).  The reference sums its
process workers' arrays the same way (chatcarlo/transport.py:416-437).
"""
from __future__ import annotations

import numpy as np

RANK_STRIDE = 1 << 40      # history-index offset per rank


def shard_range(n_histories: int, rank: int, world: int) -> tuple[int, int]:
    """(first history, count) of rank's share; the remainder goes to the first ranks."""
    base, extra = divmod(int(n_histories), int(world))
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def allreduce_grid_arrays(arrays: list[np.ndarray], device=None) -> list[np.ndarray]:
    """Sum float64/int32 numpy arrays over all ranks (in place) and return them."""
    import torch
    import torch.distributed as dist
    out = []
    for a in arrays:
        t = torch.from_numpy(np.ascontiguousarray(a))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t)
        a[...] = t.cpu().numpy()
        out.append(a)
    return out


def reduce_result(res, device=None):
    """Sum a TransportResult (grid arrays, counters, per-material sums) over ranks."""
    import torch
    import torch.distributed as dist
    g = res.grid
    if g is not None:
        arrs = [g.kerma_keV, g.h10_track_pSv_cm3]
        if g.track_uncertainty:
            arrs += [g.kerma_sum2, g.h10_sum2, g.n_batches_hit]
        allreduce_grid_arrays(arrs, device)
        cnt = torch.tensor([g.n_batches, g.n_histories], dtype=torch.int64)
        if device is not None:
            cnt = cnt.to(device)
        dist.all_reduce(cnt)
        g.n_batches, g.n_histories = (int(x) for x in cnt.cpu().tolist())
    n = torch.tensor([res.n_histories, round(res.fraction_absorbed * res.n_histories),
                      round(res.fraction_escaped * res.n_histories),
                      round(res.mean_scatter_events * res.n_histories), res.n_fluorescence],
                     dtype=torch.int64)
    if device is not None:
        n = n.to(device)
    dist.all_reduce(n)
    tot, nab, nes, nsc, nfl = (int(x) for x in n.cpu().tolist())
    res.n_histories = tot
    res.fraction_absorbed = nab / max(tot, 1)
    res.fraction_escaped = nes / max(tot, 1)
    res.mean_scatter_events = nsc / max(tot, 1)
    res.n_fluorescence = nfl
    return res
