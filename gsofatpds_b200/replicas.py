"""Host logic of multi-GPU runs: replicas only.

The fill-path search needs no data exchange between GPUs (the reference's
ranks exchange only end-of-run totals, gSoFa_SOAComparison/main.cu:43-47),
so N GPUs run N independent factorizations.  The only collectives are a
barrier around the timed region and a max over ranks of the measured time;
the throughput of the job is all ranks' work over the slowest rank's time.
These helpers run unchanged on the gloo (CPU) and nccl (GPU) backends.

A stream of independent matrices is spread over the ranks by per-rank
request queues with work stealing (StealingQueue): the reference's
(disabled) MPI stealing, gSoFa_SOAComparison/symbfact_warp_centric_new_
scheduling.cuh:3224-3485, where a rank that has finished its own chunks
fetch-and-adds a victim's head pointer (MPI_Fetch_and_op on a window) to
claim the victim's next chunk, trying victims (rank + 1 + k) mod P in turn
and moving on when the claimed index is past the victim's end.  Here the
units are whole matrices and the head pointers are counters in a
torch.distributed Store (TCPStore.add is an atomic fetch-and-add on the
host): no GPU collective is involved.
"""
import json

import torch


def max_over_ranks(value, dist=None, device="cpu"):
    """Largest `value` over all ranks (the value itself without a group)."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, steps, units_per_step, max_ms):
    """Units per second of the whole job (every rank did `steps` steps of
    `units_per_step` units; the job took the slowest rank's `max_ms`)."""
    if max_ms <= 0:
        return 0.0
    return world * steps * units_per_step / (max_ms / 1e3)


def same_input_on_all_ranks(checksum, dist=None, device="cpu"):
    """True when every rank built the same input (seeded generators)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return True
    t = torch.tensor([int(checksum) & 0x7FFFFFFFFFFFFFFF], dtype=torch.int64, device=device)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return all(int(o.item()) == int(t.item()) for o in out)


def assign_queues(costs, world):
    """Longest-first assignment: requests in decreasing cost order (ties by
    index), each to the rank with the least cost so far (ties: lowest rank).
    Returns one list of request indices per rank, largest first."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    queues = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        queues[r].append(i)
        load[r] += float(costs[i])
    return queues


class StealingQueue:
    """Per-rank request queues over a shared Store; every rank must build
    the same `queues` (a list per rank of request indices).

    Iterating yields the request indices this rank processes: its own queue
    head first, then, when its queue is exhausted, the heads of victims
    (rank + 1 + k) mod world in turn.  Each claim is one atomic add on the
    owner's head counter, so every request is yielded on exactly one rank.
    Each claim is recorded under `<prefix>/by/<index>` = the claiming rank.
    """

    def __init__(self, store, rank, world, queues, prefix="gsofa/steal"):
        if len(queues) != world:
            raise ValueError("need one queue per rank")
        self.store = store
        self.rank = rank
        self.world = world
        self.queues = [list(q) for q in queues]
        self.prefix = prefix
        self.stolen = 0

    def _claim(self, owner):
        i = int(self.store.add("%s/head/%d" % (self.prefix, owner), 1)) - 1
        q = self.queues[owner]
        if i >= len(q):
            return None
        self.store.set("%s/by/%d" % (self.prefix, q[i]), str(self.rank))
        return q[i]

    def __iter__(self):
        for k in range(self.world):
            owner = (self.rank + k) % self.world
            while True:
                req = self._claim(owner)
                if req is None:
                    break
                if owner != self.rank:
                    self.stolen += 1
                yield req

    def publish(self, req, summary):
        """Record a request's result summary (a JSON-serialisable dict)."""
        self.store.set("%s/result/%d" % (self.prefix, req), json.dumps(summary))

    def owners(self, count):
        """Claiming rank of requests 0..count-1 (waits until all are claimed)."""
        keys = ["%s/by/%d" % (self.prefix, i) for i in range(count)]
        self.store.wait(keys)
        return [int(self.store.get(k)) for k in keys]

    def results(self, count):
        """Published summaries of requests 0..count-1 (waits for all)."""
        keys = ["%s/result/%d" % (self.prefix, i) for i in range(count)]
        self.store.wait(keys)
        return [json.loads(self.store.get(k)) for k in keys]
