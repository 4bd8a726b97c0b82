"""run_transport's sharded mode on the device: two ranks (processes) that
both use cuda:0, joined by a gloo process group (the one GPU of this test
stands in for one GPU per rank; the ranks' kernels never wait on each
other, only the host-side collectives do).  Each rank runs its half of the
histories and the device grids are summed in place through
cc_grid_device_buffers; the merged result must equal a one-rank run of the
same seed and histories: the shard boundaries fall on batch boundaries, so
even the batch statistics are the same up to the order of the FP64
additions."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_HIST, BATCH, SEED = 2_000_000, 200_000, 77


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from chatcarlo_b200 import workloads as W
        from chatcarlo_b200.transport import run_transport
        g = W.make_grid(W.ROOM_GRID)
        r = run_transport(W.room(), n_histories=N_HIST, seed=SEED, batch_size=BATCH, dose_grid=True, grid=g)
        q.put((rank, g.kerma_keV, g.h10_track_pSv_cm3, g.kerma_sum2, g.n_batches_hit, g.n_batches, g.n_histories,
               r.n_histories, r.fraction_absorbed, r.n_batches, r.energy_deposited_MeV, r.energy_deposited_sem_MeV))
    finally:
        dist.destroy_process_group()


def test_two_ranks_equal_one_run():
    from chatcarlo_b200 import workloads as W
    from chatcarlo_b200.transport import run_transport
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = W.make_grid(W.ROOM_GRID)
    r = run_transport(W.room(), n_histories=N_HIST, seed=SEED, batch_size=BATCH, dose_grid=True, grid=g,
                      distributed=False)
    for rank, k, h, k2, nh, nb, nhist, n, fa, nbat, dep, sem in out:
        assert n == N_HIST and nhist == N_HIST and nb == g.n_batches == 10 and nbat == r.n_batches
        np.testing.assert_allclose(k, g.kerma_keV, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(h, g.h10_track_pSv_cm3, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(k2, g.kerma_sum2, rtol=1e-9, atol=1e-12)
        np.testing.assert_array_equal(nh, g.n_batches_hit)
        assert fa == pytest.approx(r.fraction_absorbed, abs=1e-12)
        assert set(dep) == set(r.energy_deposited_MeV)
        for m in dep:
            assert dep[m] == pytest.approx(r.energy_deposited_MeV[m], rel=1e-9)
            assert sem[m] == pytest.approx(r.energy_deposited_sem_MeV[m], rel=1e-6)
