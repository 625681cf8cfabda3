"""A batch of independent FCIDUMPs (the points of a dissociation curve)
spread over the GPUs of one node, one process per GPU.

The points share nothing while they are solved, so each rank takes its share
(point i goes to rank i mod world), solves it as one batch on its own GPU
(mcd_batch_*), and the per-point results (energy, reports, and optionally the
1- and 2-RDMs) are gathered to rank 0 over torch.distributed; there is no
collective on the data path.  The reference solves a curve one point after
another (experiments/4.4-binding-curve/dissociation.sh:2-9).

The solving step is a parameter (`solve_share`), so that the sharding and
the gather run, and are tested, without a GPU.
"""
from typing import Callable, Dict, List, Optional, Sequence


def share(n: int, rank: int, world: int) -> List[int]:
    """The points of rank `rank`: i = rank, rank + world, ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(range(rank, n, world))


def gather_results(local: Dict[int, dict], n: int, dist=None, dst: int = 0) -> Optional[List[dict]]:
    """Rank `dst` receives the results of all ranks as a list indexed by
    point (every point must be present exactly once); the others receive
    None.  Without `dist`, `local` must hold every point."""
    if dist is None:
        parts = [local]
    else:
        parts = [None] * dist.get_world_size() if dist.get_rank() == dst else None
        dist.gather_object(local, parts, dst=dst)
        if dist.get_rank() != dst:
            return None
    out: List[Optional[dict]] = [None] * n
    for part in parts:
        for i, r in part.items():
            if out[i] is not None:
                raise ValueError(f"point {i} came from two ranks")
            out[i] = r
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise ValueError(f"points {missing} came from no rank")
    return out  # type: ignore[return-value]


def batch_solver(paths: Sequence[str], with_rdm: bool = False, **options) -> Callable[[List[int]], Dict[int, dict]]:
    """The GPU solving step: the given points of `paths` as one CDFCIBatch
    with `options` (mcd_options keywords) on the current device."""

    def solve_share(points: List[int]) -> Dict[int, dict]:
        import mcdfci_b200 as mc

        if not points:
            return {}
        fc = [mc.Fcidump(paths[i]) for i in points]
        b = mc.CDFCIBatch(fc, **options)
        try:
            energies = b.solve()
            out = {}
            for j, i in enumerate(points):
                rec = {"energy": energies[j], "reports": b.reports[j]}
                out[i] = rec
        finally:
            b.close()
        if with_rdm:
            # RDMs from a single-instance solve of the same point (the batch
            # exposes energies and reports; mcd_rdm works on a solver).
            for i in points:
                s = mc.CDFCI(mc.Fcidump(paths[i]), **options)
                try:
                    out[i]["energy_single"] = s.solve()
                    g1, g2 = s.rdm()
                    out[i]["rdm1"] = g1.tolist()
                    out[i]["rdm2"] = g2.tolist()
                finally:
                    s.close()
        return out

    return solve_share


def solve_curve(n: int, solve_share: Callable[[List[int]], Dict[int, dict]], dist=None) -> Optional[List[dict]]:
    """Every rank solves its share with `solve_share(points)`; rank 0 returns
    the results of all n points in order, the other ranks None."""
    rank = dist.get_rank() if dist is not None else 0
    world = dist.get_world_size() if dist is not None else 1
    local = solve_share(share(n, rank, world))
    return gather_results(local, n, dist)
