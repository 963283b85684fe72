"""Host logic of the multi-GPU split (swpathtracer_b200/shard.py), on CPU ranks over gloo."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from swpathtracer_b200 import shard


@pytest.mark.parametrize("spp,world", [(16, 1), (16, 3), (1024, 8), (5, 8), (0, 2)])
def test_sample_split_covers_every_sample_once(spp, world):
    ranges = [shard.sample_split(spp, world, r) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == spp
    for (a, b), (c, d) in zip(ranges, ranges[1:]):
        assert b == c and a <= b
    sizes = [b - a for a, b in ranges]
    assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.sample_split(spp, world, world)


@pytest.mark.parametrize("sampler", ["jittered", "uniform"])
def test_rank_params_draw_disjoint_samples(sampler):
    from swpathtracer_b200 import scenes
    p = scenes.pt_params(spp=37, sampler=sampler, seed=5, spp_offset=3)
    seen = []
    for world in (1, 3, 4):
        spans = []
        for r in range(world):
            q = shard.rank_params(p, world, r)
            n = shard.effective_spp(q.spp, q.pixel_sampler)
            spans.append((q.spp_offset, q.spp_offset + n))
            assert q.seed == p.seed and q.path_length == p.path_length
        for (a, b), (c, d) in zip(spans, spans[1:]):
            assert b == c
        assert spans[0][0] == 3
        seen.append(sum(b - a for a, b in spans))
    assert seen[0] == shard.effective_spp(37, p.pixel_sampler)


def test_assign_jobs_is_a_partition_within_the_lpt_bound():
    rng = np.random.default_rng(3)
    costs = [shard.job_cost(int(rng.integers(128, 1024)) ** 2, 64, int(rng.integers(1000, 500000)))
             for _ in range(64)]
    for world in (1, 2, 4, 8):
        parts = shard.assign_jobs(costs, world)
        assert sorted(j for p in parts for j in p) == list(range(64))
        loads = [sum(costs[j] for j in p) for p in parts]
        lower = max(max(costs), sum(costs) / world)
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-6 * lower
    assert shard.assign_jobs([], 3) == [[], [], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        spp = 10
        a, b = shard.sample_split(spp, world, rank)
        # this rank's mean image over its samples: sample s contributes the value s everywhere
        img = torch.full((4, 3, 3), float(np.mean(np.arange(a, b))), dtype=torch.float32)
        shard.combine_images(img, b - a, spp)
        out[rank] = img.numpy().copy()
    finally:
        dist.destroy_process_group()


def test_combine_images_over_gloo_gives_the_mean_of_all_samples():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        np.testing.assert_allclose(out[r], np.mean(np.arange(10)), rtol=1e-6)
