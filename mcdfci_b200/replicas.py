"""Aggregation for N independent solver replicas, one process per GPU.

The mCDFCI iteration is a sequential chain (one block of coordinates after
another), so N GPUs run N independent replicas with no collective on the data
path.  The only collective is the one that turns per-rank timings into a
whole-job rate: each rank's timed region is reduced with a max, and the job
rate is the units all ranks processed divided by that slowest time.
"""


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The maximum of `value` over the ranks of the default process group
    (the value itself when `dist` is None)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank: float, seconds: float, world: int, dist=None, device="cpu") -> float:
    """Whole-job rate of `world` replicas that each processed
    `units_per_rank` units in `seconds` (their own timed region)."""
    slowest = max_over_ranks(seconds, dist, device)
    if slowest <= 0.0:
        raise ValueError("the timed region must be positive")
    return world * units_per_rank / slowest
