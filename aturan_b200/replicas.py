"""Multi-GPU plumbing for the path: independent replicas, one process per GPU.

The dynamical-core step has no exchange step at the 41 x 181 x 361 size (the state fits one
B200), so N GPUs run N independent replicas (weak scaling); the only collective is the max of the
per-rank device times, taken so that a multi-GPU number is the slowest rank's.
"""


def replica_seed(base, rank):
    """Each replica integrates its own seeded state."""
    return int(base) + int(rank)


def max_over_ranks(value, dist=None, device="cpu"):
    """The maximum of a per-rank float over the process group (identity without one)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(n_cells, steps, world, seconds):
    """Whole-job cell-steps per second: every rank advanced n_cells cells `steps` times."""
    return n_cells * steps * world / seconds
