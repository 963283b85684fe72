"""Multi-GPU sharding of the path: one process per GPU, no data-path collective except the final sum.

Every unit of work is independent (rays, pixel samples, whole scenes), so a job is split across ranks
and the only exchange is one sum of the fp32 accumulation images at the end:

* ``sample_split`` / ``rank_params``: the spp of one render are cut into contiguous per-rank shares;
  rank r's ``spp_offset`` starts past every sample the lower ranks take (after the square rounding of
  the regular and jittered samplers), so no two ranks draw the same Philox streams.
* ``assign_jobs``: whole scenes of a batch go to ranks by longest-processing-time-first on an estimated
  cost (paths x expected segments), the classic 4/3-approximation for makespan.
* ``combine_images``: the per-rank mean images weighted by their sample counts are summed over the
  process group (NCCL on GPUs, gloo on CPUs) into the mean over all samples.
* ``render_sharded``: the three together for one path-traced image.
"""
import heapq

import numpy as np


def sample_split(spp, world, rank):
    """[begin, end) of the samples rank `rank` of `world` renders (ranges differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    base, extra = divmod(int(spp), world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def effective_spp(spp, sampler):
    """Samples the path tracer actually takes: regular and jittered round spp up to a square
    (pixel_samplers/regular_pixel_sampler.cpp:6-7, jittered_pixel_sampler.cpp:6-7)."""
    from . import abi
    if spp <= 0:
        return 0
    if sampler == abi.PIXEL_UNIFORM:
        return int(spp)
    k = int(np.ceil(np.sqrt(float(spp))))
    return k * k


def rank_params(params, world, rank):
    """A copy of an spt_pt_params for rank `rank`: its share of the spp, and an spp_offset past every
    sample the lower ranks take, so no two ranks draw the same Philox streams."""
    import ctypes
    from . import abi
    out = abi.PtParams()
    ctypes.memmove(ctypes.byref(out), ctypes.byref(params), ctypes.sizeof(params))
    offset = params.spp_offset
    for r in range(rank):
        a, b = sample_split(params.spp, world, r)
        offset += effective_spp(b - a, params.pixel_sampler)
    a, b = sample_split(params.spp, world, rank)
    out.spp = b - a
    out.spp_offset = offset
    return out


def render_sharded(scene, cam, params, image, group=None):
    """Path-traces cam over scene with the spp split across the ranks of the process group; image (a
    cuda float tensor of h*w*3) ends up holding the mean over all ranks' samples on every rank.
    Returns (this rank's render stats, total samples per pixel)."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    mine = rank_params(params, world, rank)
    n = effective_spp(mine.spp, mine.pixel_sampler)
    total = sum(effective_spp(b - a, params.pixel_sampler)
                for a, b in (sample_split(params.spp, world, r) for r in range(world)))
    if n:
        st = scene.pathtrace_device(cam, mine, image.data_ptr())
    else:
        image.zero_()
        st = None
    combine_images(image, n, total, group)
    return st, total


def job_cost(n_pixels, spp, tris):
    """Estimated cost of a path-tracing job: paths times a traversal term growing with log(tris)."""
    return float(n_pixels) * float(spp) * (1.0 + np.log2(max(int(tris), 2)) / 8.0)


def assign_jobs(costs, world):
    """Longest processing time first: job indices per rank, each rank's list in job order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for j in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        load, r = heapq.heappop(heap)
        out[r].append(j)
        heapq.heappush(heap, (load + float(costs[j]), r))
    return [sorted(o) for o in out]


def combine_images(image, n_samples, total_samples, group=None):
    """In place: image (a torch tensor holding this rank's mean over n_samples) becomes the mean over
    all ranks' samples.  Collective: every rank of the group calls it with its own tensor."""
    import torch.distributed as dist
    if total_samples <= 0:
        raise ValueError("no samples")
    image.mul_(float(n_samples) / float(total_samples))
    dist.all_reduce(image, op=dist.ReduceOp.SUM, group=group)
    return image
