"""z-slab sharding host logic on CPU ranks (gloo, world_size 2).

Each rank runs the reference's BCLP dose pass (oracle, float64) on its slab;
the all-reduced sums must equal the single-process sums of the whole volume,
and the slab partition must cover every slice exactly once."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from vamtoolbox_b200.distributed import bclp_stats_allreduce, max_allreduce, slab_range


def test_slab_range_partitions():
    for nz in (1, 5, 256, 257):
        for world in (1, 2, 3, 8):
            if world > nz:
                continue
            cover = []
            for r in range(world):
                z0, z1 = slab_range(nz, world, r)
                assert z1 - z0 in (nz // world, nz // world + 1)
                cover += list(range(z0, z1))
            assert cover == list(range(nz))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from oracle import oracle as O

        rng = np.random.default_rng(0)
        nz = 7
        dose = rng.uniform(0, 1, (12, 12, nz))
        target = (rng.uniform(0, 1, (12, 12, nz)) > 0.5).astype(float)
        f, m, dm = O.response_tables(B=12, M=0.6)
        z0, z1 = slab_range(nz, world, rank)
        _, _, s = O.bclp_dose_pass(dose[:, :, z0:z1], target[:, :, z0:z1], f, m, dm, 0.05, 1.0, 2.0)
        st = torch.tensor(s, dtype=torch.float64)
        bclp_stats_allreduce(st)
        mx = torch.tensor([float(dose[:, :, z0:z1].max())], dtype=torch.float64)
        max_allreduce(mx)
        q.put((rank, st.numpy(), float(mx[0])))
    finally:
        dist.destroy_process_group()


def test_two_rank_stats_equal_single_process():
    from oracle import oracle as O

    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(0)
    dose = rng.uniform(0, 1, (12, 12, 7))
    target = (rng.uniform(0, 1, (12, 12, 7)) > 0.5).astype(float)
    f, m, dm = O.response_tables(B=12, M=0.6)
    _, _, ref = O.bclp_dose_pass(dose, target, f, m, dm, 0.05, 1.0, 2.0)
    for _, st, mx in res:
        assert np.allclose(st, ref, rtol=1e-12, atol=1e-12)
        assert mx == dose.max()


def _dead_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=5))
    if rank == 1:
        os._exit(0)  # leaves between steps, before the collective
    try:
        bclp_stats_allreduce(torch.zeros(9, dtype=torch.float64))
        q.put("completed")
    except Exception as exc:
        q.put(type(exc).__name__)


def test_lost_rank_surfaces_as_error_not_hang():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_dead_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert out != "completed"
