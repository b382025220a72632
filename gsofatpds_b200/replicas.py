"""Host logic of multi-GPU runs: replicas only.

The fill-path search needs no data exchange between GPUs (the reference's
ranks exchange only end-of-run totals, gSoFa_SOAComparison/main.cu:43-47),
so N GPUs run N independent factorizations.  The only collectives are a
barrier around the timed region and a max over ranks of the measured time;
the throughput of the job is all ranks' work over the slowest rank's time.
These helpers run unchanged on the gloo (CPU) and nccl (GPU) backends.
"""
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
