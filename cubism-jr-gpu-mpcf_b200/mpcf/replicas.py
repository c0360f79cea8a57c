"""Running the hot path on several GPUs: replicas, no data exchange.

The path advances one block per GPU with no inter-GPU halo exchange and no
collective on the data (one GPU per block, as the reference runs one block
per MPI rank, GridMPI.h:65-106, but without the Cartesian halo exchange).
With N ranks (one process per GPU, torch.distributed for the plumbing):

  * independent domains (an ensemble) are split across ranks by
    `partition_domains`, balanced by cell count, contiguous per rank;
  * every rank advances its own share with its own solver;
  * timing is taken on each device and reduced with MAX over ranks
    (`max_over_ranks`), the work with SUM (`sum_over_ranks`), so the reported
    throughput is all ranks' cell-stage updates over the slowest rank's time.

The only collectives are these two scalar reductions and barriers around the
timed region; nothing of the state crosses between GPUs.
"""
import numpy as np


def partition_domains(cells, world):
    """Split domain indices 0..len(cells)-1 into `world` contiguous groups of
    near-equal total cell count.  Returns a list of index lists (some may be
    empty when there are fewer domains than ranks)."""
    cells = [int(c) for c in cells]
    n = len(cells)
    if world < 1:
        raise ValueError("world must be >= 1")
    total = float(sum(cells))
    groups = [[] for _ in range(world)]
    r, acc = 0, 0.0
    for i, c in enumerate(cells):
        # move to the next rank once this one has its share, keeping at least
        # one domain for every remaining rank when there are enough domains
        remaining_domains = n - i
        remaining_ranks = world - r - 1
        if groups[r] and r < world - 1 and (acc + c / 2.0 > total * (r + 1) / world or remaining_domains <= remaining_ranks):
            r += 1
        groups[r].append(i)
        acc += c
    return groups


def max_over_ranks(dist, value, device=None):
    """MAX of a float over all ranks (identity without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value, device=None):
    """SUM of a float over all ranks (identity without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def throughput(dist, cells_this_rank, stages, ms_this_rank, device=None):
    """Whole-job cell-stage updates per second: sum of all ranks' work over
    the slowest rank's device time."""
    work = sum_over_ranks(dist, float(cells_this_rank) * stages, device)
    ms = max_over_ranks(dist, ms_this_rank, device)
    return work / (ms * 1e-3), ms
