"""spt_bvh_build_device: the device-built tree against the reference's host-built tree.

1. Layout and box rule: depth-first, left-first nodes; every primitive in exactly one leaf; the root
   box is the union of the primitive boxes and every other box is its primitives' union inflated by
   1e-3, bit for bit (the rule of acceleration/sbvh.cpp:409-412 the traversals rely on).
2. Closest hits: t bit-exact with the reference tree's on every ray; the primitive differs only
   where two primitives are hit at the same t.
3. Deterministic, and correct on degenerate inputs (one primitive, coincident primitives, spheres).
"""
import numpy as np
import pytest

import swpathtracer_b200 as spt
from swpathtracer_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def prim_boxes(packed):
    """Primitive boxes as the reference computes them (primitives/triangle.cpp, sphere.cpp)."""
    types, data = packed.types, packed.data
    v = data.reshape(-1, 3, 3)
    mn, mx = v.min(axis=1), v.max(axis=1)
    sph = types == abi.PRIM_SPHERE
    if sph.any():
        c, r = data[sph, :3], data[sph, 3:4]
        mn[sph], mx[sph] = c - r, c + r
    return mn, mx


def check_layout_and_boxes(nodes, refs, n, mn, mx):
    assert sorted(refs.tolist()) == list(range(n))
    first = np.zeros(len(nodes), np.int64)
    last = np.zeros(len(nodes), np.int64)
    for i in range(len(nodes) - 1, -1, -1):   # children follow their parent in depth-first order
        nd = nodes[i]
        if nd["count"]:
            first[i], last[i] = nd["right"], nd["right"] + nd["count"]
        else:
            r = int(nd["right"])
            assert i + 1 < r < len(nodes)
            assert last[i + 1] == first[r]
            first[i], last[i] = first[i + 1], last[r]
    assert first[0] == 0 and last[0] == n
    pmn, pmx = mn[refs], mx[refs]
    eps = np.float32(1e-3)
    for i, nd in enumerate(nodes):
        umn = pmn[first[i]:last[i]].min(axis=0)
        umx = pmx[first[i]:last[i]].max(axis=0)
        if i:
            umn, umx = umn - eps, umx + eps
        assert np.array_equal(np.asarray(nd["min"], np.float32).view(np.uint32), umn.view(np.uint32)), i
        assert np.array_equal(np.asarray(nd["max"], np.float32).view(np.uint32), umx.view(np.uint32)), i


def compare_hits(device, packed, rays, max_tie_fraction=1e-4):
    ref_scene = spt.GpuScene(device, packed)
    dev_bvh = spt.Bvh(packed, device=device)
    dev_scene = spt.GpuScene(device, packed, dev_bvh)
    a = ref_scene.intersect(rays)["hits"]
    b = dev_scene.intersect(rays)["hits"]
    assert np.array_equal(a["t"].view(np.uint32), b["t"].view(np.uint32))
    same = a["prim_id"] == b["prim_id"]
    assert (1.0 - same.mean()) <= max_tie_fraction
    assert np.array_equal(a["u"][same].view(np.uint32), b["u"][same].view(np.uint32))
    assert np.array_equal(a["v"][same].view(np.uint32), b["v"][same].view(np.uint32))
    return dev_bvh


@pytest.mark.parametrize("builder", [lambda: scenes.displaced_mesh_scene(5), lambda: scenes.box_scene(4),
                                     lambda: scenes.furnace_scene("lambertian")])
def test_device_tree_layout_boxes_and_hits(device, builder):
    sb = builder()
    packed = sb.build()
    rays = scenes.incoherent_rays(1 << 16, seed=51, half_extent=1.5)
    bvh = compare_hits(device, packed, rays)
    nodes, refs = bvh.export()
    n = packed.n_prims
    mn, mx = prim_boxes(packed)
    check_layout_and_boxes(nodes, refs, n, mn, mx)
    st = bvh.statistics()
    assert st.num_references == n and st.num_unreferenced == 0
    assert st.num_nodes == len(nodes) and st.tree_height + 2 <= 64
    assert st.max_prims_leaf <= 8 and st.build_ms > 0


def test_device_tree_is_deterministic(device):
    packed = scenes.displaced_mesh_scene(6).build()
    n1, r1 = spt.Bvh(packed, device=device).export()
    n2, r2 = spt.Bvh(packed, device=device).export()
    assert n1.tobytes() == n2.tobytes() and np.array_equal(r1, r2)


def test_device_tree_on_degenerate_inputs(device):
    rng = np.random.default_rng(5)
    tri = np.array([[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]], np.float32)
    rays = np.zeros((4096, 8), np.float32)
    rays[:, 0:2] = rng.uniform(-0.2, 1.0, (4096, 2))
    rays[:, 2] = 1.0
    rays[:, 6] = -1.0
    for copies in (1, 2, 37, 1000):
        sb = scenes.SceneBuilder()
        m = sb.material(sb.layered_bsdf(sb.lambertian()))
        sb.triangles(np.repeat(tri, copies, axis=0), m)
        packed = sb.build()
        # every copy is hit at the same t: the tie may pick another copy, never another t
        bvh = compare_hits(device, packed, rays, max_tie_fraction=1.0)
        nodes, refs = bvh.export()
        mn, mx = prim_boxes(packed)
        check_layout_and_boxes(nodes, refs, copies, mn, mx)
