"""Runs with one process per GPU: replica bookkeeping.

The benchmark system (one 48^3 box) is a single elimination forest that this
library factors on one GPU; a run on N GPUs is N independent replicas (no data
exchange on the factor or solve path).  Many independent systems (a forest of
boxes) shard by system instead.  What the ranks share is bookkeeping only:

* ``max_over_ranks`` - a time measured on every rank, reduced to the slowest
  (the job takes as long as its slowest replica);
* ``shard`` - the systems a rank owns (round robin, every system exactly once);
* ``whole_job_rate`` - units processed by all ranks divided by that time.

The reduction runs over the process group given (NCCL on GPUs, gloo on CPU).
"""


def max_over_ranks(value, dist=None, device='cpu'):
    """Maximum of a per-rank float over the default process group (or itself)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(count, rank, world):
    """Indices of the units (systems) that rank owns: rank, rank + world, ..."""
    if not 0 <= rank < world:
        raise ValueError('rank %d outside a world of %d' % (rank, world))
    return list(range(rank, count, world))


def whole_job_rate(units_per_rank, world, seconds):
    """Aggregate throughput: every rank processed units_per_rank in at most seconds."""
    if seconds <= 0:
        raise ValueError('time must be positive')
    return world * units_per_rank / seconds
