"""Independent replicas on several GPUs (one process per GPU, no data-path
collective): the whole-job rate is the units every rank processed over the
slowest rank's time, taken with one all-reduce (MAX) over the ranks' own device
timings.  Used by the benchmark's N-GPU runs; any torch.distributed backend."""


def max_over_ranks(x, dist=None, device="cpu"):
    """Largest value of x over the ranks of the default process group (x itself when
    no group is initialised)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, seconds, world, dist=None, device="cpu"):
    """(whole-job units per second, slowest rank's seconds) for `world` replicas that
    each processed units_per_rank units in their own `seconds`."""
    slowest = max_over_ranks(seconds, dist, device)
    return units_per_rank * world / slowest, slowest
