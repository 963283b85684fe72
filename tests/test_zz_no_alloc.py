"""spt_intersect_noalloc (include/spt_noalloc.h) against spt_intersect on the same rays.

Collected last on purpose: the entry point's static device buffer is shared by the whole process,
so this file also checks that it works after every other test has run (and alone).
"""
import numpy as np
import pytest
import torch

import swpathtracer_b200 as spt
from swpathtracer_b200 import abi, scenes

pytestmark = pytest.mark.gpu

MAX_RAYS = 1 << 16


def _same(a, b):
    assert a["hits"].tobytes() == b["hits"].tobytes()
    np.testing.assert_array_equal(a["tests"], b["tests"])
    np.testing.assert_array_equal(a["nhits"], b["nhits"])


@pytest.mark.parametrize("builder", [lambda: scenes.displaced_mesh_scene(5), lambda: scenes.furnace_scene("coating")])
def test_noalloc_matches_intersect_on_two_calls_in_a_row(device, builder):
    gs = spt.GpuScene(device, builder().build())
    first = scenes.incoherent_rays(MAX_RAYS, seed=41, half_extent=1.5)
    second = scenes.incoherent_rays(12345, seed=42, half_extent=1.5)
    expect1 = gs.intersect(first, counts=True)
    expect2 = gs.intersect(second, counts=True)
    got1 = gs.intersect_noalloc(first, counts=True)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    got2 = gs.intersect_noalloc(second, counts=True)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    _same(got1, expect1)
    _same(got2, expect2)
    assert free_after == free_before
    # without the count outputs: the same hits
    assert gs.intersect_noalloc(second)["hits"].tobytes() == expect2["hits"].tobytes()


def test_noalloc_rejects_batches_beyond_its_buffer(device):
    gs = spt.GpuScene(device, scenes.box_scene(2).build())
    rays = scenes.incoherent_rays(MAX_RAYS + 1, seed=43, half_extent=1.0)
    with pytest.raises(spt.SptError) as e:
        gs.intersect_noalloc(rays)
    assert e.value.status == abi.SPT_ERR_INVALID_ARGUMENT
    assert "65536" in str(e.value)
    assert gs.intersect_noalloc(rays[:0])["hits"].shape == (0,)
    # a rejected call leaves the entry point usable
    _same(gs.intersect_noalloc(rays[:100], counts=True), gs.intersect(rays[:100], counts=True))
