"""Pins the oracle (the project's CPU restatement) before it is trusted as the GPU checker.

* against the committed golden fixtures made from the reference's own code (tests/golden),
* against the published Philox-4x32-10 known-answer vectors,
* and, where the reference sources were compiled here (oracle/_ref), live against the reference.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from swpathtracer_b200 import abi, scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "golden.json")) as f:
    META = json.load(f)

BUILDERS = {
    "box_icosphere": (lambda: scenes.box_scene(3), lambda: scenes.box_camera(64, 48)),
    "displaced_mesh": (lambda: scenes.displaced_mesh_scene(5), lambda: scenes.displaced_mesh_camera(80, 45)),
    "furnace_spheres": (lambda: scenes.furnace_scene("coating"), lambda: scenes.furnace_camera(48, 48)),
    "smooth_mesh": (lambda: scenes.smooth_mesh_scene(3), lambda: scenes.box_camera(64, 48)),
}


def _scene_hash(p):
    h = hashlib.sha256()
    for a in (p.types, p.data, p.normals, p.mats):
        if a is not None:
            h.update(a.tobytes())
    return h.hexdigest()


def _tree_hash(nodes, refs):
    h = hashlib.sha256()
    h.update(nodes.tobytes())
    h.update(refs.tobytes())
    return h.hexdigest()


def test_philox_known_answers(oracle):
    for kat in META["philox_kat"]:
        got = oracle.philox(kat["ctr"], kat["key"])
        assert [int(x) for x in got] == kat["out"]


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_generators_are_stable(name):
    packed = BUILDERS[name][0]().build()
    assert packed.n_prims == META["scenes"][name]["n_prims"]
    assert _scene_hash(packed) == META["scenes"][name]["scene_sha256"]


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_oracle_tree_matches_reference_golden(oracle, name):
    g = META["scenes"][name]
    osc = oracle.scene(BUILDERS[name][0]().build())
    nodes, refs = osc.tree()
    assert _tree_hash(nodes, refs) == g["tree_sha256"]
    st = osc.tree_stats()
    for k, v in g["tree_stats"].items():
        assert getattr(st, k) == v, k


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_oracle_intersect_matches_reference_golden(oracle, name):
    fx = np.load(os.path.join(GOLDEN, name + ".npz"))
    osc = oracle.scene(BUILDERS[name][0]().build())
    r = osc.intersect(fx["rays"])
    np.testing.assert_array_equal(r["hits"]["prim_id"], fx["prim"])
    np.testing.assert_array_equal(r["hits"]["t"].view(np.uint32), fx["t"].view(np.uint32))
    np.testing.assert_array_equal(r["normals"].view(np.uint32), fx["normals"].view(np.uint32))
    np.testing.assert_array_equal(r["tests"], fx["tests"])
    np.testing.assert_array_equal(r["nhits"], fx["nhits"])


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_oracle_raycast_matches_reference_golden(oracle, name):
    fx = np.load(os.path.join(GOLDEN, name + ".npz"))
    mk, mkcam = BUILDERS[name]
    osc = oracle.scene(mk().build())
    cam = mkcam()
    normal, st = osc.raycast(cam, abi.RAYCAST_NORMAL)
    depth, _ = osc.raycast(cam, abi.RAYCAST_DEPTH)
    count, _ = osc.raycast(cam, abi.RAYCAST_COUNT)
    np.testing.assert_array_equal(normal.view(np.uint32), fx["img_normal"].view(np.uint32))
    np.testing.assert_array_equal(depth.view(np.uint32), fx["img_depth"].view(np.uint32))
    np.testing.assert_array_equal(count, fx["img_count"].astype(np.int64))
    for k, v in META["scenes"][name]["raycast_stats"].items():
        assert getattr(st, k) == v, k


def test_oracle_depth_and_count_postprocess(oracle):
    """Depth normalisation (depth_raycaster.cpp:9-34) and the HSL heat map (int_test_count_raycaster.cpp:20-73)."""
    depth = np.array([[-1.0, 2.0], [4.0, 3.0]], np.float32)
    rgb = oracle.depth_to_rgb(depth)
    np.testing.assert_allclose(rgb[..., 0], [[0.0, 0.0], [1.0, 0.5]])
    cnt = np.array([[0, 10], [5, 10]], np.int64)
    heat = oracle.count_to_rgb(cnt, 0, 10)
    assert np.allclose(heat[0, 0], [0.0, 0.0, 0.0])  # t = 0: lightness 0 -> black
    assert heat[0, 1, 0] > 0.9 and heat[0, 1, 2] < 0.1  # t = 1: hue 0 -> red


# ---- live comparison with the reference's own code (only where oracle/_ref was built) ----------

LIVE = {
    "box_icosphere": lambda: scenes.box_scene(4),
    "layered_box": lambda: scenes.layered_box_scene(4),
    "smooth_mesh": lambda: scenes.smooth_mesh_scene(4),
    "furnace_lambertian": lambda: scenes.furnace_scene("lambertian"),
}


@pytest.mark.parametrize("name", sorted(LIVE))
def test_oracle_matches_reference_live(ref_harness, oracle, name):
    packed = LIVE[name]().build()
    rs = ref_harness.scene(packed)
    osc = oracle.scene(packed)
    n1, r1 = rs.tree()
    n2, r2 = osc.tree()
    assert n1.tobytes() == n2.tobytes() and r1.tobytes() == r2.tobytes()
    ext = 11.0 if name.startswith("furnace") else 3.2
    rays = scenes.incoherent_rays(20000, seed=19, half_extent=ext)
    a, b = rs.intersect(rays), osc.intersect(rays)
    assert a["hits"].tobytes() == b["hits"].tobytes()
    np.testing.assert_array_equal(a["tests"], b["tests"])
    np.testing.assert_array_equal(a["nhits"], b["nhits"])
    np.testing.assert_array_equal(a["normals"].view(np.uint32), b["normals"].view(np.uint32))


def test_no_accel_matches_reference_live(ref_harness, oracle):
    sb = scenes.box_scene(2)
    sb.accel = abi.ACCEL_NONE
    packed = sb.build()
    rays = scenes.incoherent_rays(5000, seed=2, half_extent=1.0)
    a = ref_harness.scene(packed).intersect(rays)
    b = oracle.scene(packed).intersect(rays)
    assert a["hits"].tobytes() == b["hits"].tobytes()
    np.testing.assert_array_equal(a["tests"], b["tests"])


@pytest.mark.parametrize("kind", ["pinhole", "orthographic"])
def test_camera_rays_match_reference_live(ref_harness, oracle, kind):
    from oracle.bindings import camera_rays
    if kind == "pinhole":
        cam = scenes.camera("pinhole", position=(0.3, 1.2, 4.0), look_at=(0.1, -0.2, 0.0), up=(0.1, 1.0, 0.0),
                            fov=47.5, width=97, height=61)
    else:
        cam = scenes.camera("orthographic", position=(2.0, 1.0, 6.0), look_at=(0, 0, 0), width=64, height=40,
                            window=(-1.7, 1.3, -0.9, 1.1))
    np.testing.assert_array_equal(camera_rays(cam, ref_harness).view(np.uint32), oracle.camera_rays(cam).view(np.uint32))


def test_bsdf_walk_statistics_match_reference_live(ref_harness, oracle):
    """Material::evalBSDF: the oracle's layered walk (Philox draws) and the reference's (mt19937
    draws) agree in distribution: mean f*cos/pdf per outgoing direction within Monte Carlo error."""
    packed = scenes.furnace_scene("coating").build()
    rs = ref_harness.scene(packed)
    osc = oracle.scene(packed)
    n = 200000
    rng = np.random.default_rng(4)
    for wy in (0.9, 0.4, -0.6):
        wo = np.zeros((n, 3), np.float32)
        wo[:, 0] = np.sqrt(1 - wy * wy)
        wo[:, 1] = wy
        a = rs.eval_material(1, wo, seed=3)
        b = osc.eval_material(1, wo, seed=3, path0=0, depth=0)
        wa = a[:, 0] * a[:, 8] / a[:, 6]
        wb = b[:, 0] * b[:, 8] / b[:, 6]
        se = np.sqrt(wa.var() / n + wb.var() / n)
        assert abs(wa.mean() - wb.mean()) < 5 * se + 1e-6, (wy, wa.mean(), wb.mean())
    del rng
