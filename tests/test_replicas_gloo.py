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


def _steal_worker(rank, world, port, q, queues, costs_ms):
    import time
    from gsofatpds_b200 import replicas
    from datetime import timedelta
    store = dist.TCPStore("127.0.0.1", port, world, rank == 0, timeout=timedelta(seconds=60))
    sq = replicas.StealingQueue(store, rank, world, queues)
    store.add("gsofa/steal/ready", 1)  # start together
    while int(store.add("gsofa/steal/ready", 0)) < world:
        time.sleep(0.005)
    done = []
    t0 = time.perf_counter()
    for req in sq:
        time.sleep(costs_ms[req] / 1e3)
        sq.publish(req, {"req": req, "rank": rank})
        done.append(req)
    busy = time.perf_counter() - t0
    owners = sq.owners(len(costs_ms))
    res = sq.results(len(costs_ms))
    store.add("gsofa/steal/exit", 1)
    if rank == 0:  # the store's server lives in rank 0: wait for every reader
        store.wait(["gsofa/steal/exit"])
        while int(store.add("gsofa/steal/exit", 0)) < world:
            time.sleep(0.01)
    q.put((rank, done, sq.stolen, busy, owners, [r["rank"] for r in res]))


def _run_steal(world, queues, costs_ms):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_steal_worker, args=(r, world, port, q, queues, costs_ms))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in range(world)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def test_work_stealing_every_request_exactly_once():
    """Every request lands in rank 0's queue; the idle ranks steal from its
    head (victims rank+1+k), and each request is processed exactly once."""
    world = 3
    costs = [30.0] * 12
    res = _run_steal(world, [list(range(12)), [], []], costs)
    done = [set(r[1]) for r in res]
    assert set().union(*done) == set(range(12))
    assert sum(len(d) for d in done) == 12
    assert res[1][2] > 0 and res[2][2] > 0  # ranks 1 and 2 stole
    assert res[0][2] == 0
    for rank, d, _, _, owners, published in res:
        for req in d:
            assert owners[req] == rank and published[req] == rank
    # balanced by stealing: rank 0 alone would do all 12; with two thieves
    # no rank does much more than its share of 4 (slack for a loaded host)
    assert max(len(d) for d in done) <= 8


def test_longest_first_queues():
    from gsofatpds_b200 import replicas
    costs = [5, 1, 9, 3, 3, 7, 2]
    qs = replicas.assign_queues(costs, 3)
    assert sorted(i for q in qs for i in q) == list(range(7))
    loads = [sum(costs[i] for i in q) for q in qs]
    assert max(loads) - min(loads) <= max(costs)
    assert qs[0][0] == 2 and qs[1][0] == 5  # largest first, lowest rank on ties
    assert replicas.assign_queues([], 2) == [[], []]
