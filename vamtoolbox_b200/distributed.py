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


def gather_zslabs(local, nz_total: int, group=None):
    """The whole [..., nz_total] array from every rank's z-slab [..., z0:z1] (slab_range): the slabs, padded to
    the largest slab, are all-gathered and concatenated in rank order on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    z0, z1 = slab_range(nz_total, world, rank)
    if local.shape[-1] != z1 - z0:
        raise ValueError(f"rank {rank}: slab of {local.shape[-1]} slices, expected {z1 - z0}")
    zmax = max(b - a for a, b in (slab_range(nz_total, world, r) for r in range(world)))
    pad = torch.zeros(local.shape[:-1] + (zmax,), dtype=local.dtype, device=local.device)
    pad[..., : z1 - z0] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad.contiguous(), group=group)
    return torch.cat([parts[r][..., : b - a] for r, (a, b) in
                      enumerate(slab_range(nz_total, world, r) for r in range(world))], dim=-1)


def optimize_bclp_zslab(target_geo, proj_geo, options, group=None, gather=True):
    """optimize(target_geo, proj_geo, options) for BCLP (vamtoolbox/optimize.py:174-217 ->
    vamtoolbox/optimizer/BCLP.py) over z-slabs, one per rank of ``group`` (one process per GPU, NCCL).

    Parallel beam without inclination treats slices independently in every projection, so each rank
    builds its own projector on slices [z0, z1) of the target (slab_range) and runs the device engine
    there; the 9 loss / norm sums are all-reduced every iteration, so every rank takes the whole volume's
    loss, gradient scale and convergence decision, as one process would (float32 sums combined in another
    order).  Returns (Sinogram, Reconstruction, loss) of the whole volume on every rank when ``gather``
    (the slabs all-gathered), else this rank's slabs (sinogram [nR, nA, z1 - z0], dose [nY, nX, z1 - z0]).
    The caller's geometry objects are not modified."""
    import copy

    import torch
    import torch.distributed as dist

    from . import geometry
    from .optimizer.BCLP import BCLPNorm

    if options.method != "BCLP":
        raise ValueError("optimize_bclp_zslab runs BCLP")
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    arr = np.atleast_3d(np.asarray(target_geo.array))
    nz = arr.shape[2]
    z0, z1 = slab_range(nz, world, rank)
    if z1 <= z0:
        raise ValueError(f"{world} ranks for {nz} slices: rank {rank} has no slice")
    tg, pg = copy.copy(target_geo), copy.copy(proj_geo)
    tg.array = np.ascontiguousarray(arr[:, :, z0:z1])
    if options.units != "normalized" or pg.absorption_coeff is not None:
        pg.calcAbsorptionMask(tg)
    bclp = BCLPNorm(tg, pg, options)
    if not bclp._device_init_ok():
        raise ValueError("optimize_bclp_zslab needs the device engine on a parallel-beam projector")
    g = bclp.checkSinogramShape(bclp.gradientDescentDevice(graph=False,
                                                           reduce_stats=lambda s: bclp_stats_allreduce(s, group)),
                                "cylindrical")
    if not gather:
        return g, bclp.dose, bclp.logs.loss
    dev = bclp.P.device
    g_all = gather_zslabs(torch.as_tensor(g, device=dev), nz, group).cpu().numpy()
    d_all = gather_zslabs(torch.as_tensor(bclp.dose, device=dev), nz, group).cpu().numpy()
    return (geometry.Sinogram(g_all, proj_geo, options), geometry.Reconstruction(d_all, proj_geo, options),
            bclp.logs.loss)
