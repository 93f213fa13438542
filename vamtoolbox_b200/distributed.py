"""Multi-GPU plumbing: z-slabs for the parallel beam, angles for the ray
tracer, targets for batched multi-target runs.

Parallel beam: with no inclination, z-slices are independent in the forward
projector, both backprojectors and every elementwise step
(vamtoolbox/projector/Projector3DParallel.py:132,176), so a volume splits into
contiguous z-slabs, one per rank, with no exchange in any projection.  The
only coupling is global scalars: the BCLP loss / norm sums (BCLP.py:332-437)
and the max / VER normalisations of CAL and OSMO (CAL.py:177, OSMO.py:60,68).

Ray tracer: rays bend in z, so slabs are not independent; each rank traces the
rays of a contiguous block of angles through replicas of the medium fields.
The forward (integrate) of a rank fills its own sinogram rows, with no
exchange; the deposit of a rank is a partial dose grid, summed over ranks
(the dose is linear in the rays, and the absorption weighting that follows
the deposit is elementwise).  With the dose replicated, the dose pass is the
same on every rank and a rank updates only its own sinogram rows, so a
sharded ray-traced BCLP iteration exchanges one dose grid.

Multi-target: independent targets are assigned to ranks whole (no exchange).

One process per GPU, torch.distributed over NCCL (gloo on CPU for tests).
"""
from __future__ import annotations

import numpy as np


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


def angle_range(n_angles: int, world: int, rank: int):
    """[a0, a1) of rank's contiguous block of angles (the ray tracer's shard)."""
    return slab_range(n_angles, world, rank)


def ray_indices(n_det: int, n_angles: int, n_z: int, a0: int, a1: int):
    """Flat ray / sinogram indices of the angles [a0, a1) in the tracer's ray order,
    meshgrid(detector, angle, z, indexing="ij") (pyTorchRayTrace.py:1629-1632): ray (d, a, z) is
    (d * n_angles + a) * n_z + z.  The rays a rank traces for angles [a0, a1) are these, in this order."""
    d = np.arange(n_det)[:, None, None]
    a = np.arange(a0, a1)[None, :, None]
    z = np.arange(n_z)[None, None, :]
    return ((d * n_angles + a) * n_z + z).ravel()


def shard_angles(proj_geo, world: int, rank: int):
    """A shallow copy of ``proj_geo`` whose ``angles`` are rank's block (the projector a rank builds
    from it traces exactly the rays ``ray_indices`` names)."""
    import copy

    a0, a1 = angle_range(len(proj_geo.angles), world, rank)
    g = copy.copy(proj_geo)
    g.angles = np.asarray(proj_geo.angles)[a0:a1]
    g.n_angles = a1 - a0
    return g


def dose_allreduce(dose, group=None):
    """Sum the ranks' partial deposits in place (the one exchange of a sharded ray-traced iteration)."""
    import torch.distributed as dist

    dist.all_reduce(dose, op=dist.ReduceOp.SUM, group=group)
    return dose


def target_shards(costs, world: int):
    """Assign independent targets to ranks: longest first to the least loaded rank (ties to the lower
    rank), deterministic.  costs: estimated time per target (e.g. voxels x angles).  Returns one list
    of target indices per rank, each in ascending order."""
    if world <= 0:
        raise ValueError("bad world")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += float(costs[i])
        out[r].append(i)
    return [sorted(o) for o in out]
