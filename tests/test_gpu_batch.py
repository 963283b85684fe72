"""Batched rendering of uneven scenes in one wavefront, and the autotuner."""
import numpy as np
import pytest
import torch

import swpathtracer_b200 as spt
from swpathtracer_b200 import scenes

pytestmark = pytest.mark.gpu


def _small_batch(n=5):
    return scenes.batched_scenes(n=n, seed=7, min_tris=500, max_tris=20000, min_res=24, max_res=64, spp=4)


def test_batch_equals_individual_renders(device):
    batch = _small_batch()
    jobs, bufs = [], []
    for sb, cam, p, _ in batch:
        gs = spt.GpuScene(device, sb.build())
        jobs.append((gs, cam, p))
        bufs.append(torch.zeros(cam.height * cam.width * 3, dtype=torch.float32, device="cuda"))
    stats = spt.render_batch(device, jobs, [b.data_ptr() for b in bufs])
    torch.cuda.synchronize()
    for (gs, cam, p), b, st in zip(jobs, bufs, stats):
        single, _ = gs.pathtrace(cam, p)
        got = b.cpu().numpy().reshape(cam.height, cam.width, 3)
        np.testing.assert_allclose(got, single, rtol=1e-5, atol=1e-6)
        assert st.paths == cam.width * cam.height * p.spp


def test_tuning_does_not_change_images(device):
    batch = _small_batch(3)
    jobs = [(spt.GpuScene(device, sb.build()), cam, p) for sb, cam, p, _ in batch]
    outs = []
    for trav, cap, shade, srt in ((2, 1 << 20, 128, 2), (1, 4096, 64, 1), (0, 100000, 256, 0), (1, 1 << 20, 128, 1)):
        t = spt.default_tune()
        t.traversal, t.capacity, t.shade_block, t.sort_shading = trav, cap, shade, srt
        bufs = [torch.zeros(c.height * c.width * 3, dtype=torch.float32, device="cuda") for _, c, _ in jobs]
        spt.render_batch(device, jobs, [b.data_ptr() for b in bufs], tune=t)
        outs.append([b.cpu().numpy() for b in bufs])
    for other in outs[1:]:
        for a, b in zip(outs[0], other):
            np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6)


def test_autotune_and_cache(device, tmp_path):
    batch = _small_batch(4)
    jobs = [(spt.GpuScene(device, sb.build()), cam, p) for sb, cam, p, _ in batch]
    cache = str(tmp_path / "tune.txt")
    t1 = spt.autotune(device, jobs, cache)
    assert t1.capacity in (1 << 20, 1 << 21, 1 << 22) and t1.traversal in (0, 1, 2)
    assert open(cache).read().count("\n") == 1
    t2 = spt.autotune(device, jobs, cache)  # from the cache
    assert bytes(t1) == bytes(t2)
