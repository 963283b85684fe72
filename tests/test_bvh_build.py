"""The product's host SAH builder (libspt_cuda.so, spt_bvh_build) against the oracle's tree.

Host code only: runs without a GPU.  The trees must be identical node for node (boxes, links,
leaf order) whatever the thread count, since the GPU's hit-count mode and equal-t tie breaks
depend on the exact tree.
"""
import numpy as np
import pytest

import swpathtracer_b200 as spt
from swpathtracer_b200 import abi, scenes

CASES = {
    "box_icosphere": lambda: scenes.box_scene(4),
    "displaced_mesh": lambda: scenes.displaced_mesh_scene(6),
    "layered_box": lambda: scenes.layered_box_scene(5),
    "smooth_mesh": lambda: scenes.smooth_mesh_scene(4),
    "furnace": lambda: scenes.furnace_scene("plastic"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tree_identical_to_oracle(oracle, name):
    packed = CASES[name]().build()
    nodes, refs = spt.Bvh(packed).export()
    onodes, orefs = oracle.scene(packed).tree()
    assert nodes.tobytes() == onodes.tobytes()
    assert refs.tobytes() == orefs.tobytes()


def test_thread_count_invariance():
    packed = scenes.displaced_mesh_scene(7).build()
    trees = [spt.Bvh(packed, n_threads=t).export() for t in (1, 3, 8)]
    for n, r in trees[1:]:
        assert n.tobytes() == trees[0][0].tobytes() and r.tobytes() == trees[0][1].tobytes()


def test_statistics_match_oracle(oracle):
    packed = scenes.box_scene(5).build()
    a = spt.Bvh(packed).statistics()
    b = oracle.scene(packed).tree_stats()
    for f in ("num_nodes", "num_inner_nodes", "num_leaf_nodes", "tree_height", "min_prims_leaf",
              "max_prims_leaf", "num_references", "num_unreferenced"):
        assert getattr(a, f) == getattr(b, f), f


def test_tree_invariants():
    packed = scenes.box_scene(4).build()
    nodes, refs = spt.Bvh(packed).export()
    assert sorted(refs.tolist()) == list(range(packed.n_prims))  # every primitive in exactly one leaf
    leaf = nodes["count"] > 0
    assert nodes["count"][leaf].sum() == packed.n_prims
    inner = np.nonzero(~leaf)[0]
    for i in inner[:2000]:
        for c in (i + 1, nodes["right"][i]):
            # children are contained in the parent except below the root (inflated by 1e-3 only)
            if i > 0:
                assert (nodes["min"][c] >= nodes["min"][i]).all() and (nodes["max"][c] <= nodes["max"][i]).all()


def test_degenerate_inputs(oracle):
    """Many identical triangles (all centroid ties) and a single primitive."""
    sb = scenes.SceneBuilder()
    m = sb.material(sb.layered_bsdf(sb.lambertian()))
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    sb.triangles(np.repeat(tri[None], 300, 0), m)
    packed = sb.build()
    nodes, refs = spt.Bvh(packed).export()
    onodes, orefs = oracle.scene(packed).tree()
    assert nodes.tobytes() == onodes.tobytes() and refs.tobytes() == orefs.tobytes()
    sb = scenes.SceneBuilder()
    m = sb.material(sb.layered_bsdf(sb.lambertian()))
    sb.sphere((0, 0, 0), 1.0, m)
    nodes, refs = spt.Bvh(sb.build()).export()
    assert len(nodes) == 1 and nodes["count"][0] == 1
