"""Multi-rank host logic (replicas) with two gloo ranks on CPU."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from gsofatpds_b200 import gen, replicas
        n, rp, col = gen.random_extra(3000, 3, seed=1)
        chk = int(np.bitwise_xor.reduce(col.astype(np.int64) * 2654435761 + np.arange(col.size)))
        same = replicas.same_input_on_all_ranks(chk, dist)
        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
        dist.barrier()
        mx = replicas.max_over_ranks(local_ms, dist)
        value = replicas.job_throughput(world, 3, 1000.0, mx)
        q.put((rank, same, mx, value))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_throughput():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, same, mx, value in res:
        assert same
        assert mx == 150.0
        assert abs(value - 2 * 3 * 1000.0 / 0.150) < 1e-6


def test_single_process_defaults():
    from gsofatpds_b200 import replicas
    assert replicas.max_over_ranks(12.5) == 12.5
    assert replicas.job_throughput(1, 2, 10.0, 1000.0) == 20.0
    assert replicas.same_input_on_all_ranks(7)
