"""Scene scripts rendered through the front end (swpathtracer_b200/frontend.py) on the GPU: the Lua
scene equals the same scene built directly, and the saved image files match the host-side writer."""
import os

import numpy as np
import pytest

import swpathtracer_b200 as spt
from swpathtracer_b200 import abi, frontend, scenes

pytestmark = pytest.mark.gpu
SCRIPT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lua", "small_box.lua")


def _direct_scene():
    """tests/lua/small_box.lua written with SceneBuilder."""
    sb = scenes.SceneBuilder(background=(0, 0, 0))

    def matte(c):
        return sb.material(sb.layered_bsdf(sb.lambertian(kd=c)))
    grey, red, green = matte((0.75, 0.75, 0.75)), matte((0.63, 0.06, 0.05)), matte((0.14, 0.45, 0.09))
    light = sb.material(sb.layered_bsdf(sb.lambertian(kd=(0, 0, 0))), emission=(15, 15, 15))
    metal = sb.material(sb.layered_bsdf(sb.cook_torrance(roughness=0.3,
                                                         reflectance_at_normal_incidence=(0.95, 0.64, 0.54))))
    quads = [([0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], grey), ([0, 0, 1], [1, 0, 1], [1, 0, 0], [0, 0, 0], grey),
             ([0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1], grey), ([0, 0, 1], [0, 0, 0], [0, 1, 0], [0, 1, 1], red),
             ([1, 0, 0], [1, 0, 1], [1, 1, 1], [1, 1, 0], green)]
    y, lo, hi = 0.999, 0.375, 0.625
    quads.append(([lo, y, lo], [lo, y, hi], [hi, y, hi], [hi, y, lo], light))
    tris, mats = [], []
    for a, b, c, d, m in quads:
        tris += [[a, b, c], [a, c, d]]
        mats += [m, m]
    sb.triangles(np.array(tris, np.float32), np.array(mats, np.uint32))
    sb.sphere((0.5, 0.3, 0.5), 0.3, metal)
    for i in range(1, 4):
        sb.sphere((0.2 * i, 0.08, 0.85), 0.07, matte((0.2 * i, 0.5, 1 - 0.2 * i)))
    return sb.build()


@pytest.mark.parametrize("mode", ["depth", "normal", "intersection-test-count"])
def test_lua_scene_ray_casts_like_the_direct_scene(device, oracle, mode, tmp_path):
    s = frontend.load_lua(SCRIPT, globals={"INTEGRATOR": mode})
    img, st = frontend.render(s, device)
    gs = spt.GpuScene(device, _direct_scene())
    exp, est = gs.raycast(s.camera, s.raycast_mode, stats=True)
    np.testing.assert_array_equal(np.asarray(img).view(np.uint8), np.asarray(exp).view(np.uint8))
    out = tmp_path / "img.ppm"
    frontend.save(s, device, img, str(out))
    vals = np.array([int(v) for v in out.read_text().split()[4:]])
    assert len(vals) == 3 * 48 * 40
    if mode == "depth":
        rgb = oracle.depth_to_rgb(img)
    elif mode == "intersection-test-count":
        rgb = oracle.count_to_rgb(img, est.min_tests_pp, est.max_tests_pp)
    else:
        rgb = np.where(np.any(img != 0, axis=2, keepdims=True), img * np.float32(0.5) + np.float32(0.5), 0)
    spt.write_ppm(str(tmp_path / "host.ppm"), rgb.astype(np.float32), srgb=False)
    host = np.array([int(v) for v in (tmp_path / "host.ppm").read_text().split()[4:]])
    np.testing.assert_array_equal(vals, host)


def test_lua_scene_path_traces_like_the_direct_scene(device, tmp_path):
    s = frontend.load_lua(SCRIPT)
    img, st = frontend.render(s, device)
    gs = spt.GpuScene(device, _direct_scene())
    exp, _ = gs.pathtrace(s.camera, s.pt_params)
    np.testing.assert_allclose(img, exp, rtol=1e-5, atol=1e-6)
    assert st.paths == 48 * 40 * 16
    out = tmp_path / "pt.ppm"
    frontend.save(s, device, img, str(out))
    assert out.read_text().startswith("P3\n48 40\n255\n")
