"""Parity at the benchmark configuration itself, on the CPU: the 1,310,720-triangle displaced
icosphere of the headline workload.

The fixtures (tests/golden/c1_mesh.npz, configs.json) come from the reference's own SBVH::build and
SBVH::intersect (acceleration/sbvh.cpp:12-37, 478-510) run by tests/golden/make_golden_configs.py.
Here the product's host SAH builder must reproduce the reference's tree node for node at full size,
and the oracle must reproduce the reference's hits and test counts on the sampled headline rays.
The GPU side of the same pins is in tests/test_gpu_config_pins.py.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import swpathtracer_b200 as spt
from swpathtracer_b200 import abi, scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "configs.json")) as f:
    CONFIGS = json.load(f)


def _tree_hash(nodes, refs):
    h = hashlib.sha256()
    h.update(nodes.tobytes())
    h.update(refs.tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def c1_packed():
    return scenes.displaced_mesh_scene(8).build()


@pytest.fixture(scope="module")
def c1_rays():
    """The sampled rays of the headline batch: scenes.incoherent_rays(2^24, seed=1)[index]."""
    fx = np.load(os.path.join(GOLDEN, "c1_mesh.npz"))
    return fx["index"], scenes.incoherent_rays(1 << 24, seed=1)[fx["index"]]


def test_c1_host_tree_is_the_reference_tree(c1_packed):
    g = CONFIGS["c1"]
    assert c1_packed.n_prims == g["n_prims"] == 1310720
    bvh = spt.Bvh(c1_packed)
    nodes, refs = bvh.export()
    assert _tree_hash(nodes, refs) == g["tree_sha256"]
    st = bvh.statistics()
    for k, v in g["tree_stats"].items():
        assert getattr(st, k) == v, k
    bvh.close()


def test_c1_oracle_hits_match_reference_sample(oracle, c1_packed, c1_rays):
    fx = np.load(os.path.join(GOLDEN, "c1_mesh.npz"))
    _, rays = c1_rays
    osc = oracle.scene(c1_packed)
    r = osc.intersect(rays, n_threads=os.cpu_count() or 1, want_normals=False)
    np.testing.assert_array_equal(r["hits"]["prim_id"], fx["prim"])
    hit = fx["prim"] != abi.SPT_MISS
    np.testing.assert_array_equal(r["hits"]["t"][hit].view(np.uint32), fx["t"][hit].view(np.uint32))
    np.testing.assert_array_equal(r["tests"], fx["tests"])
    np.testing.assert_array_equal(r["nhits"], fx["nhits"])
    # the sample is a meaningful one: hits and misses, and deep traversals
    assert 0.1 < hit.mean() < 0.6 and fx["tests"].max() > 200
    osc.close()
