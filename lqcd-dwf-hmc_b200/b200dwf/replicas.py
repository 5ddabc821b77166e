"""Replica bookkeeping for runs on several GPUs of one node.

The hot path does not shard (one lattice per GPU, no data-path exchange):
`bench.py --gpus N` runs N independent replicas, one process per GPU.  Across
ranks only two things happen, both here: a barrier around the timed region and
the max-over-ranks of the timed duration, from which the whole-job throughput
is formed.  The functions take the torch.distributed module (NCCL on GPUs,
gloo in the CPU tests) or None for a single process.
"""


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(seconds, dist, device="cpu"):
    """The slowest rank's duration (every rank gets the same value)."""
    if dist is None:
        return float(seconds)
    import torch
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, seconds_max, world):
    """Aggregate throughput of `world` replicas that each processed
    `units_per_rank` units, timed as the slowest rank."""
    if seconds_max <= 0.0:
        raise ValueError("non-positive duration")
    return world * units_per_rank / seconds_max
