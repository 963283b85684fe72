"""The 8-wide collapse (swpathtracer_b200/csrc/wide_build.cpp) checked on the host, without a GPU.

tests/wide_check.cpp builds the reference's SAH tree and its 8-wide collapse for a scene and checks
that every triangle lands in exactly one wide leaf, that child and triangle indices are in range,
that every quantized child box contains the reference boxes below it (what the wide traversal's
exactness needs), and that the collapse is deterministic (it builds the root's subtrees on several
threads).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from swpathtracer_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "swpathtracer_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("wide") / "wide_check")
    cmd = [gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-pthread", "-I" + CSRC, os.path.join(HERE, "wide_check.cpp"),
           os.path.join(CSRC, "bvh_build.cpp"), os.path.join(CSRC, "wide_build.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def _check(checker, tmp_path, tris):
    tris = np.ascontiguousarray(np.asarray(tris, np.float32).reshape(-1, 9))
    path = tmp_path / "scene.bin"
    with open(path, "wb") as f:
        f.write(np.uint32(tris.shape[0]).tobytes())
        f.write(tris.tobytes())
    r = subprocess.run([checker, str(path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok")
    return r.stdout.split()


def _triangles(sb):
    types, data, _, _ = sb.arrays()
    assert (types == 0).all()
    return data


@pytest.mark.parametrize("name,make", [
    ("displaced mesh, 20,480 tris", lambda: _triangles(scenes.displaced_mesh_scene(5))),
    ("displaced mesh, 327,680 tris", lambda: _triangles(scenes.displaced_mesh_scene(7))),
    ("box scene", lambda: _triangles(scenes.box_scene(4))),
    ("window room", lambda: _triangles(scenes.window_room_scene(0.1))),
])
def test_collapse_invariants(checker, tmp_path, name, make):
    _check(checker, tmp_path, make())


@pytest.mark.parametrize("copies", [1, 2, 3, 25, 37, 1000])
def test_collapse_of_coincident_triangles(checker, tmp_path, copies):
    # one large reference leaf: it becomes chunks of three, or wide nodes of its own when too large
    tri = np.array([[0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0]], np.float32)
    out = _check(checker, tmp_path, np.repeat(tri, copies, axis=0))
    assert int(out[2]) == copies


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_collapse_of_random_triangles(checker, tmp_path, seed):
    rng = np.random.default_rng(seed)
    n = [500, 7000, 40000][seed]
    centres = rng.uniform(-10, 10, (n, 1, 3))
    tris = centres + rng.normal(0, 0.3 * (seed + 1), (n, 3, 3))
    _check(checker, tmp_path, tris)
