"""Ray queries and ray-cast integrators on the GPU against the oracle, bit for bit.

The oracle (oracle/spt_oracle.cpp) restates the reference's traversal exactly and is pinned to
the reference's own code (tests/test_oracle_pins.py, tests/golden).  Hit/miss, primitive id,
t, u/v-derived normals and the per-ray test counts must all match exactly.
"""
import numpy as np
import pytest

from swpathtracer_b200 import abi, scenes
import swpathtracer_b200 as spt

pytestmark = pytest.mark.gpu

SCENES = {
    "box_icosphere": lambda: scenes.box_scene(4),
    "displaced_mesh": lambda: scenes.displaced_mesh_scene(6),
    "furnace_spheres": lambda: scenes.furnace_scene("coating"),
    "layered_box": lambda: scenes.layered_box_scene(5),
}


def _rays_for(name, n=1 << 15):
    ext = 12.0 if name == "furnace_spheres" else 2.0
    return scenes.incoherent_rays(n, seed=7, half_extent=ext)


@pytest.mark.parametrize("name", sorted(SCENES))
def test_intersect_matches_oracle(device, oracle, name):
    packed = SCENES[name]().build()
    gs = spt.GpuScene(device, packed)
    osc = oracle.scene(packed)
    rays = _rays_for(name)
    got = gs.intersect(rays, counts=True)
    exp = osc.intersect(rays)
    np.testing.assert_array_equal(got["hits"]["prim_id"], exp["hits"]["prim_id"])
    hit = exp["hits"]["prim_id"] != abi.SPT_MISS
    np.testing.assert_array_equal(got["hits"]["t"][hit].view(np.uint32), exp["hits"]["t"][hit].view(np.uint32))
    np.testing.assert_array_equal(got["tests"], exp["tests"])
    np.testing.assert_array_equal(got["nhits"], exp["nhits"])


@pytest.mark.parametrize("name", ["box_icosphere", "displaced_mesh", "furnace_spheres"])
@pytest.mark.parametrize("mode", [abi.RAYCAST_NORMAL, abi.RAYCAST_DEPTH, abi.RAYCAST_COUNT])
def test_raycast_modes_match_oracle(device, oracle, name, mode):
    packed = SCENES[name]().build()
    if name == "furnace_spheres":
        cam = scenes.furnace_camera(96, 80)
    elif name == "displaced_mesh":
        cam = scenes.displaced_mesh_camera(160, 90)
    else:
        cam = scenes.box_camera(128, 96)
    gs = spt.GpuScene(device, packed)
    osc = oracle.scene(packed)
    got, gst = gs.raycast(cam, mode, stats=True)
    exp, est = osc.raycast(cam, mode)
    if mode == abi.RAYCAST_COUNT:
        np.testing.assert_array_equal(got, exp)
    else:
        np.testing.assert_array_equal(got.view(np.uint32), exp.view(np.uint32))
    for f in ("int_tests", "int_hits", "min_tests_pp", "max_tests_pp", "min_hits_pp", "max_hits_pp"):
        assert getattr(gst, f) == getattr(est, f), f


def test_no_accel_structure(device, oracle):
    sb = scenes.box_scene(2)
    sb.accel = abi.ACCEL_NONE
    packed = sb.build()
    gs = spt.GpuScene(device, packed)
    osc = oracle.scene(packed)
    rays = scenes.incoherent_rays(4096, seed=3, half_extent=1.0)
    got = gs.intersect(rays, counts=True)
    exp = osc.intersect(rays)
    np.testing.assert_array_equal(got["hits"]["prim_id"], exp["hits"]["prim_id"])
    np.testing.assert_array_equal(got["tests"], exp["tests"])
    np.testing.assert_array_equal(got["nhits"], exp["nhits"])


def test_empty_and_ragged_batches(device, oracle):
    packed = scenes.box_scene(2).build()
    gs = spt.GpuScene(device, packed)
    osc = oracle.scene(packed)
    for n in (0, 1, 31, 33, 1000, 4097):
        rays = scenes.incoherent_rays(max(n, 1), seed=n + 1, half_extent=1.0)[:n]
        got = gs.intersect(rays, counts=True)
        assert got["hits"].shape == (n,)
        if n:
            exp = osc.intersect(rays)
            np.testing.assert_array_equal(got["hits"]["prim_id"], exp["hits"]["prim_id"])
            np.testing.assert_array_equal(got["tests"], exp["tests"])


def test_full_size_mesh_closest_equals_exhaustive(device):
    """1,310,720 triangles, 2^24 incoherent rays: the ordered, pruned traversal returns exactly the
    hit of the reference-order exhaustive traversal for every ray (a size-independent property of
    the two GPU kernels).  The comparison of a sample of the same rays with the reference's own
    hits is test_gpu_config_pins.py::test_c1_headline_rays_match_reference."""
    import torch
    packed = scenes.displaced_mesh_scene(8).build()
    gs = spt.GpuScene(device, packed)
    n = 1 << 24
    rays = torch.from_numpy(scenes.incoherent_rays(n, seed=1)).cuda()
    hits = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    ref_hits = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    gs.intersect_device(rays.data_ptr(), n, hits.data_ptr(), 0)
    gs.count_device(rays.data_ptr(), n, ref_hits.data_ptr(), None, None)
    torch.cuda.synchronize()
    assert torch.equal(hits[:, :2], ref_hits[:, :2]), "ordered traversal differs from the reference order"
    h = hits.cpu().numpy()
    prim = h[:, 1].view(np.uint32)
    t = h[:, 0].view(np.float32)
    hit = prim != abi.SPT_MISS
    assert (prim[hit] < packed.n_prims).all()
    assert (t[hit] > 0).all() and np.isinf(t[~hit]).all()
    assert 0.1 < hit.mean() < 0.6


def test_pipelined_host_queries_match_device_queries(device):
    """spt_intersect with page-locked host buffers runs in chunks over four streams; the hits and
    counts equal one device-side query of the whole batch (and the pageable path)."""
    import torch
    packed = scenes.displaced_mesh_scene(6).build()
    gs = spt.GpuScene(device, packed)
    n = (1 << 21) * 2 + 12345                   # five chunks of 2^20, the last one partial
    rays = scenes.incoherent_rays(n, seed=77, half_extent=1.5)
    h_rays = torch.from_numpy(rays).pin_memory()
    h_hits = torch.empty((n, 4), dtype=torch.int32).pin_memory().numpy().view(abi.HIT_DTYPE).reshape(n)
    got = gs.intersect(h_rays.numpy(), out=h_hits)
    d_rays = torch.from_numpy(rays).cuda()
    d_hits = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    gs.intersect_device(d_rays.data_ptr(), n, d_hits.data_ptr(), 0)
    torch.cuda.synchronize()
    assert got["hits"].tobytes() == d_hits.cpu().numpy().tobytes()
    # counts through the pipeline against the pageable (single-stream) path on a slice
    sub = rays[: (1 << 21) + 999]
    m = sub.shape[0]
    pinned = torch.from_numpy(np.ascontiguousarray(sub)).pin_memory().numpy()
    p_hits = torch.empty((m, 4), dtype=torch.int32).pin_memory().numpy().view(abi.HIT_DTYPE).reshape(m)
    p_tests = torch.empty(m, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    p_nh = torch.empty(m, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    a = gs.intersect(pinned, out=p_hits, out_counts=(p_tests, p_nh))
    b = gs.intersect(np.ascontiguousarray(sub), counts=True)
    assert a["hits"].tobytes() == b["hits"].tobytes()
    np.testing.assert_array_equal(a["tests"], b["tests"])
    np.testing.assert_array_equal(a["nhits"], b["nhits"])


def test_coherence_order_keeps_every_hit(device):
    """A batch of at least 2^21 rays is traced in coherence order (entry point into the root box, then
    direction; misses last) and its hits go back to each ray's own index.  Against the same rays in
    calls below that size (their own order), bit for bit, on a batch whose keys reach every edge:
    axis-aligned directions (zero components), origins inside the root box, rays that miss it, and
    both ray layouts."""
    import torch
    packed = scenes.displaced_mesh_scene(6).build()
    gs = spt.GpuScene(device, packed)
    n = (1 << 21) + 17
    rays = scenes.incoherent_rays(n, seed=79, half_extent=1.5)
    axes = np.eye(3, dtype=np.float32)
    k = np.arange(60000)
    rays[k, 4:7] = axes[k % 3] * np.where(k % 2, 1.0, -1.0)[:, None]       # axis-aligned directions
    rays[60000:90000, 0:3] *= 0.3                                           # origins inside the box
    d_rays = torch.from_numpy(rays).cuda()
    ordered = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    plain = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    gs.intersect_device(d_rays.data_ptr(), n, ordered.data_ptr(), 0)
    half = n // 2                                                           # both calls below 2^21
    gs.intersect_device(d_rays.data_ptr(), half, plain.data_ptr(), 0)
    gs.intersect_device(d_rays[half:].data_ptr(), n - half, plain[half:].data_ptr(), 0)
    torch.cuda.synchronize()
    assert torch.equal(ordered, plain)
    # the three stages one by one: the order is a permutation with its inverse, and the hits in that
    # order are the rays' hits
    order = torch.empty(2 * n + 1, dtype=torch.int32, device="cuda")
    in_order = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    back = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    gs.ray_order_device(d_rays.data_ptr(), n, order.data_ptr(), 0)
    gs.intersect_ordered_device(d_rays.data_ptr(), order.data_ptr(), n, in_order.data_ptr(), 0)
    gs.hits_unorder_device(order.data_ptr(), n, in_order.data_ptr(), back.data_ptr(), 0)
    torch.cuda.synchronize()
    m = int(order[2 * n].item())
    perm = order[:m].long()
    inv = order[n:2 * n]
    placed = inv != -1                                   # 0xFFFFFFFF: the root box test rejects the ray
    assert int(placed.sum().item()) == m
    idx = torch.arange(n, device="cuda")
    assert torch.equal(torch.sort(perm).values, idx[placed])
    assert torch.equal(perm[inv[placed].long()], idx[placed])
    assert torch.equal(in_order[:m], plain[perm]) and torch.equal(back, plain)
    assert (plain[~placed][:, 1] == -1).all()            # every ray without a place misses
    miss = ordered[:, 1].cpu().numpy().view(np.uint32) == abi.SPT_MISS
    assert 0.2 < miss.mean() < 0.9
    # the reference's 24-byte layout through the pageable path, ordered as well
    rays6 = np.ascontiguousarray(np.concatenate([rays[:, 0:3], rays[:, 4:7]], axis=1))
    assert gs.intersect(rays6)["hits"].tobytes() == ordered.cpu().numpy().tobytes()


def test_coherence_order_on_spheres_and_unsupported_scenes(device, oracle):
    """The ordered path on a sphere scene (the 8-wide tree's sphere leaves) equals the oracle on a
    sample and the batch's own order everywhere; a scene without the persistent traversal (no
    acceleration structure) keeps its own order in spt_intersect_device and refuses the ordered
    stage with SPT_ERR_UNSUPPORTED."""
    import torch
    from swpathtracer_b200.native import SptError
    packed = scenes.furnace_scene("coating").build()
    gs = spt.GpuScene(device, packed)
    n = (1 << 21) + 5
    rays = scenes.incoherent_rays(n, seed=80, half_extent=12.0)
    d_rays = torch.from_numpy(rays).cuda()
    ordered = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    plain = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    gs.intersect_device(d_rays.data_ptr(), n, ordered.data_ptr(), 0)
    half = n // 2
    gs.intersect_device(d_rays.data_ptr(), half, plain.data_ptr(), 0)
    gs.intersect_device(d_rays[half:].data_ptr(), n - half, plain[half:].data_ptr(), 0)
    torch.cuda.synchronize()
    assert torch.equal(ordered, plain)
    exp = oracle.scene(packed).intersect(rays[:20000])
    got = ordered[:20000].cpu().numpy()
    np.testing.assert_array_equal(got[:, 1].view(np.uint32), exp["hits"]["prim_id"])
    sb = scenes.box_scene(2)
    sb.accel = abi.ACCEL_NONE
    flat = spt.GpuScene(device, sb.build())
    order = torch.empty(2 * n + 1, dtype=torch.int32, device="cuda")
    flat.ray_order_device(d_rays.data_ptr(), n, order.data_ptr(), 0)      # the order itself is defined
    with pytest.raises(SptError):
        flat.intersect_ordered_device(d_rays.data_ptr(), order.data_ptr(), n, ordered.data_ptr(), 0)
    m = 50000
    flat.intersect_device(d_rays.data_ptr(), m, plain.data_ptr(), 0)
    torch.cuda.synchronize()
    exp = oracle.scene(sb.build()).intersect(rays[:m])
    np.testing.assert_array_equal(plain[:m, 1].cpu().numpy().view(np.uint32), exp["hits"]["prim_id"])


def test_reference_ray_layout_matches_padded_layout(device):
    """spt_intersect_packed takes rays as the reference's Ray lies in memory (origin then direction,
    24 bytes): the same hits and counts as the padded layout, on the pageable path, the pipelined
    page-locked path (chunks of 2^20 rays, the last partial) and an empty batch."""
    import torch
    packed = scenes.displaced_mesh_scene(6).build()
    gs = spt.GpuScene(device, packed)
    n = (1 << 21) + 4321
    rays8 = scenes.incoherent_rays(n, seed=78, half_extent=1.5)
    rays6 = np.ascontiguousarray(np.concatenate([rays8[:, 0:3], rays8[:, 4:7]], axis=1))
    small8, small6 = rays8[:50000], np.ascontiguousarray(rays6[:50000])
    a = gs.intersect(small8, counts=True)
    b = gs.intersect(small6, counts=True)
    assert a["hits"].tobytes() == b["hits"].tobytes()
    np.testing.assert_array_equal(a["tests"], b["tests"])
    np.testing.assert_array_equal(a["nhits"], b["nhits"])
    h6 = torch.from_numpy(rays6).pin_memory().numpy()
    h_hits = torch.empty((n, 4), dtype=torch.int32).pin_memory().numpy().view(abi.HIT_DTYPE).reshape(n)
    got = gs.intersect(h6, out=h_hits)
    assert got["hits"].tobytes() == gs.intersect(rays8)["hits"].tobytes()
    assert gs.intersect(rays6[:0])["hits"].shape == (0,)
