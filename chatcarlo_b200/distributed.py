"""History sharding over ranks and the one tally exchange.

Histories are independent: rank r of W simulates its own contiguous range
of history indices (disjoint Philox counters, so no two ranks share a
stream) and keeps a private FP64 grid.  The single exchange step is a sum of
the tally arrays, the statistics arrays, the per-material moments and the
counters over ranks with torch.distributed (NCCL on GPUs, gloo on CPUs).
The reference sums its process workers' results the same way, in worker
order (chatcarlo/transport.py:397-437); a sum over ranks is one collective.

Under torchrun, ``run_transport`` shards by itself: every rank runs its
share of the histories on its own GPU, the device-resident grids are summed
in place by NCCL (no host round trip), and every rank returns the whole
run's result.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

RANK_STRIDE = 1 << 40      # history-index offset per rank


def shard_range(n_histories: int, rank: int, world: int) -> tuple[int, int]:
    """(first history, count) of rank's share; the remainder goes to the first ranks."""
    base, extra = divmod(int(n_histories), int(world))
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def world_info() -> tuple[int, int]:
    """(rank, world size) of the initialised default process group, else (0, 1)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def allreduce_grid_arrays(arrays: list[np.ndarray], device=None) -> list[np.ndarray]:
    """Sum float64/int32 host arrays over all ranks (in place) and return them."""
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


class _DeviceArray:
    """A device allocation of the engine seen through __cuda_array_interface__
    (so torch wraps it without a copy)."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_grid_tensors(dg) -> dict:
    """Torch views (no copies) of a DeviceGrid's device-resident totals,
    sums of squares and hit counts, plus its counts."""
    import torch
    from . import _native as N
    tot, q, nh = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nvox, nb, nhist = C.c_int64(), C.c_int64(), C.c_int64()
    N.check(dg.lib.cc_grid_device_buffers(dg.handle, C.byref(tot), C.byref(q), C.byref(nh), C.byref(nvox),
                                          C.byref(nb), C.byref(nhist)), dg.lib)
    dev = torch.device("cuda", dg.engine.device)
    out = {"totals": torch.as_tensor(_DeviceArray(tot.value, (nvox.value, 2), "<f8"), device=dev),
           "n_batches": int(nb.value), "n_histories": int(nhist.value)}
    if q.value:
        out["sum2s"] = torch.as_tensor(_DeviceArray(q.value, (nvox.value, 2), "<f8"), device=dev)
        out["n_batches_hit"] = torch.as_tensor(_DeviceArray(nh.value, (nvox.value,), "<i4"), device=dev)
    return out


def allreduce_device_grid(dg) -> None:
    """Sum a DeviceGrid over ranks in place on the devices: one all-reduce
    per array (FP64 totals and sums of squares, int32 hit counts) and one of
    the batch / history counts."""
    import torch
    import torch.distributed as dist
    t = device_grid_tensors(dg)
    for k in ("totals", "sum2s", "n_batches_hit"):
        if k in t:
            dist.all_reduce(t[k])
    cnt = torch.tensor([t["n_batches"], t["n_histories"]], dtype=torch.int64, device=t["totals"].device)
    dist.all_reduce(cnt)
    torch.cuda.synchronize(t["totals"].device)
    nb, nhist = (int(x) for x in cnt.tolist())
    from . import _native as N
    N.check(dg.lib.cc_grid_set_counts(dg.handle, nb, nhist), dg.lib)


def reduce_result(res, device=None, grid: bool = True):
    """Sum a TransportResult over ranks: counters, energy deposited per
    material with its batch moments (standard and relative errors
    recomputed from the merged moments, as transport.py:420-437,451-458),
    and, with ``grid``, the host grid's arrays."""
    import torch
    import torch.distributed as dist
    from .tally import ScalarMoments
    g = res.grid
    if grid and g is not None:
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
                      round(res.mean_scatter_events * res.n_histories), res.n_fluorescence, res.n_batches],
                     dtype=torch.int64)
    if device is not None:
        n = n.to(device)
    dist.all_reduce(n)
    tot, nab, nes, nsc, nfl, nbat = (int(x) for x in n.cpu().tolist())
    # per-material sums: every rank contributes the union of the names (a
    # rank whose histories left no energy in a material has no entry)
    names: list = [None] * dist.get_world_size()
    mom = res.moments
    mine = set(res.energy_deposited_MeV) | (set(mom.sums) if mom is not None else set())
    dist.all_gather_object(names, sorted(mine))
    keys = sorted(set().union(*map(set, names)))
    has_mom = torch.tensor([1 if mom is not None else 0], dtype=torch.int64)
    if device is not None:
        has_mom = has_mom.to(device)
    dist.all_reduce(has_mom, op=dist.ReduceOp.MIN)
    with_mom = bool(has_mom.item())
    v = np.zeros((3 if with_mom else 1, len(keys)))
    for j, k in enumerate(keys):
        v[0, j] = res.energy_deposited_MeV.get(k, 0.0)
        if with_mom:
            v[1, j] = mom.sums.get(k, 0.0)
            v[2, j] = mom.sum2s.get(k, 0.0)
    tv = torch.from_numpy(v)
    if device is not None:
        tv = tv.to(device)
    dist.all_reduce(tv)
    v = tv.cpu().numpy()
    res.n_histories = tot
    res.fraction_absorbed = nab / max(tot, 1)
    res.fraction_escaped = nes / max(tot, 1)
    res.mean_scatter_events = nsc / max(tot, 1)
    res.n_fluorescence = nfl
    res.n_batches = nbat
    res.energy_deposited_MeV = {k: float(v[0, j]) for j, k in enumerate(keys) if v[0, j] != 0.0}
    if with_mom:
        merged = ScalarMoments()
        used = [j for j in range(len(keys)) if v[1, j] != 0.0 or v[2, j] != 0.0]
        merged.add_moments({keys[j]: float(v[1, j]) for j in used}, {keys[j]: float(v[2, j]) for j in used},
                           nbat, tot)
        res.moments = merged
        res.energy_deposited_sem_MeV = {k: s / 1000.0 for k, s in merged.standard_errors().items()}
        res.energy_deposited_rel_err = merged.relative_errors()
    return res
