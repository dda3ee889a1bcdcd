"""Running one case per GPU: the timing a multi-GPU run reports.

Blocks shard naturally across GPUs, with one halo exchange per stage
(the reference's MPI exchange, peregrine/multiblock/collections/exchange/).
This build runs replicas: every rank steps its own copy of the workload and
no data crosses GPUs.  A run's time is the slowest rank's, and its
throughput is every rank's cells over that time (weak scaling).
"""


def max_over_ranks(value, dist=None, device=None):
    """The largest of a float over the ranks of the default process group."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_throughput(cells_per_rank, stages, steps, ms, world):
    """Cell-stage updates per second of the whole job: every rank's work over the slowest rank's time."""
    return cells_per_rank * stages * steps * world / (ms / 1e3)
