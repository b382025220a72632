"""Per-rank request queues with work stealing, on the device.

Two processes, each with its own context on the same GPU, drain the shared
queues of a mix of small matrices.  Their factorizations are independent (no
kernel of one waits on the other's), so sharing one GPU stands in for two
replicas.  Every matrix must be factored exactly once, with the oracle's
answer, and the idle rank must steal.
"""
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _requests():
    from gsofatpds_b200 import gen
    reqs = []
    for i in range(10):
        n = 800 + 400 * i
        reqs.append(gen.random_banded(n, bw=4 + i, extra=1 + i % 3, seed=20 + i)[1:])
    for side in (30, 45, 60):
        reqs.append(gen.grid_nd((side, side), "5")[1:])
    return reqs


def _worker(rank, world, port, q, queues):
    import time
    from datetime import timedelta
    import torch.distributed as dist
    from gsofatpds_b200 import Context, replicas
    store = dist.TCPStore("127.0.0.1", port, world, rank == 0, timeout=timedelta(seconds=120))
    reqs = _requests()
    sq = replicas.StealingQueue(store, rank, world, queues, prefix="gpu/steal")
    with Context(0) as ctx:
        store.add("gpu/steal/ready", 1)
        while int(store.add("gpu/steal/ready", 0)) < world:
            time.sleep(0.005)
        for req in sq:
            m = ctx.load_rowptr(*reqs[req])
            r = ctx.factor(m)
            c = r.counts
            sq.publish(req, {"rank": rank, "fill": int(c["fill_count"]), "nnz_l": int(c["nnz_l"]),
                             "nnz_u": int(c["nnz_u"])})
            r.close()
            m.close()
    res = sq.results(len(reqs))
    store.add("gpu/steal/exit", 1)
    if rank == 0:
        while int(store.add("gpu/steal/exit", 0)) < world:
            time.sleep(0.01)
    q.put((rank, sq.stolen, res))


def test_two_replicas_steal_and_match_oracle():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import torch.multiprocessing as mp
    from gsofatpds_b200.gen import csr_to_beg_end
    from oracle import oracle as O
    reqs = _requests()
    world = 2
    queues = [list(range(len(reqs))), []]  # everything starts on rank 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, queues)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[1][1] > 0, "rank 1 stole nothing"
    res = out[0][2]
    assert res == out[1][2]
    # rank 1's own queue is empty: everything it factored was stolen
    assert sum(1 for r in res if r["rank"] == 1) == out[1][1]
    assert out[0][1] == 0
    for i, (rp, col) in enumerate(reqs):
        b, e = csr_to_beg_end(rp)
        ref = O.rows(b, e, col)
        assert res[i]["fill"] == int(ref["fills"].sum()), i
        assert res[i]["nnz_l"] == int(ref["nnzL"].sum()), i
        assert res[i]["nnz_u"] == int(ref["nnzU"].sum()), i
