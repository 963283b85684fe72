"""Multi-GPU sharding of the path: one process per GPU, no data-path collective except the final sum.

Every unit of work is independent (rays, pixel samples, whole scenes), so a job is split across ranks
and the only exchange is one sum of the fp32 accumulation images at the end:

* ``sample_split``: the spp of one render are cut into contiguous per-rank ranges; rank r renders its
  range with ``spp_offset`` at the range's start, so its Philox streams are those samples' streams and
  no two ranks draw the same numbers.
* ``assign_jobs``: whole scenes of a batch go to ranks by longest-processing-time-first on an estimated
  cost (paths x expected segments), the classic 4/3-approximation for makespan.
* ``combine_images``: the per-rank mean images weighted by their sample counts are summed over the
  process group (NCCL on GPUs, gloo on CPUs) into the mean over all samples.
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
