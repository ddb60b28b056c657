"""Several GPUs: the path does not shard (every stage of one triangulation is
global: flips, insertions and the spectrum sort see the whole mesh), so N
processes, one per GPU, run N independent copies of the workload ("replicas
only", weak scaling).  There is no data-path collective: the ranks meet only
to time the job, which takes as long as its slowest rank (device-timed on
each rank, then the maximum over ranks after a barrier), and the job's
throughput counts every rank's units."""


def max_over_ranks(value, dist=None, device="cpu"):
    """The maximum of `value` over all ranks of `dist` (a torch.distributed
    module with an initialised process group; None: this process alone),
    after a barrier.  Every rank gets the result."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, units_per_rank, max_ms):
    """Units per second of the whole job: every rank's units over the slowest
    rank's time."""
    if max_ms <= 0:
        raise ValueError("job time must be positive")
    return world * units_per_rank / (max_ms / 1e3)
