"""The multi-GPU bench path on CPU: two gloo ranks run independent replicas (no data-path collective).

Each rank picks its own seeded sources, times its work, and the job time is the max over ranks; the whole-job
GTEPS counts every rank's traversals.
"""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    deg = np.ones(1 << 12, np.int64)
    deg[::3] = 0
    src = bench.rank_sources(deg, 16, 1, rank)
    my_seconds = 1.0 + rank  # rank 1 is the slow replica
    t = bench.max_over_ranks(my_seconds, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, src.tolist())
    if rank == 0:
        out.put((t, gathered, bench.job_gteps(32, 1000, world, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, gathered, gteps = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert t == 2.0  # max over ranks
    a, b = (np.array(x) for x in gathered)
    assert len(a) == len(b) == 16 and not np.array_equal(a, b)  # independent replicas
    assert all(x % 3 != 0 for x in np.concatenate([a, b]))  # nonzero out-degree only
    assert abs(gteps - 2 * 32 * 1000 / 2.0 / 1e9) < 1e-15


def test_single_rank_is_identity():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_gteps(10, 100, 1, 2.0) == 10 * 100 / 2.0 / 1e9
