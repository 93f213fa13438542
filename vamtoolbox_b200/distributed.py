"""Multi-GPU plumbing for z-slab sharding of the parallel-beam path.

With no inclination, z-slices are independent in the forward projector, both
backprojectors and every elementwise step (vamtoolbox/projector/Projector3DParallel.py:132,176),
so a volume splits into contiguous z-slabs, one per rank, with no exchange in
any projection.  The only coupling is global scalars: the BCLP loss / norm
sums (BCLP.py:332-437) and the max / VER normalisations of CAL and OSMO
(CAL.py:177, OSMO.py:60,68).  One process per GPU, torch.distributed over
NCCL (gloo on CPU for tests).
"""
from __future__ import annotations


def slab_range(nz_total: int, world: int, rank: int):
    """[z0, z1) of rank's contiguous slab; slabs differ in size by at most one slice."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad world / rank")
    base, extra = divmod(nz_total, world)
    z0 = rank * base + min(rank, extra)
    return z0, z0 + base + (1 if rank < extra else 0)


def bclp_stats_allreduce(stats, group=None):
    """All-reduce the 9 BCLP sums in place: entries 0-6 are sums, 7-8 maxima."""
    import torch.distributed as dist

    dist.all_reduce(stats[:7], op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(stats[7:], op=dist.ReduceOp.MAX, group=group)
    return stats


def max_allreduce(x, group=None):
    import torch.distributed as dist

    dist.all_reduce(x, op=dist.ReduceOp.MAX, group=group)
    return x
