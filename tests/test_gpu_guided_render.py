"""Guided path tracing (one-sample MIS of the learned mixture and the BSDF sampler) on the GPU.

1. Unbiased: a guided render converges to the plain path tracer's image (image and block means within
   their noise), and at an equal sample count its error against a high-sample plain render is lower
   than the plain one's on a room lit through a small window and on a scene of the 64-scene batch set.
2. A scene whose only guidable material is black (a kd = 0 light) renders as the plain tracer does:
   the guided kernels draw the same streams for the non-guidable vertices.
3. The guide trains on the render's own paths: its step count grows by at most max_steps.
"""
import numpy as np
import pytest
import torch

import swpathtracer_b200 as spt
from swpathtracer_b200 import scenes

pytestmark = pytest.mark.gpu


def relmse(a, b):
    return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))


def _render(gs, cam, p, guide=None):
    img = torch.zeros(cam.width * cam.height * 3, dtype=torch.float32, device="cuda")
    st = gs.pathtrace_guided_device(cam, p, guide, img.data_ptr()) if guide else \
        gs.pathtrace_device(cam, p, img.data_ptr())
    torch.cuda.synchronize()
    return img.cpu().numpy().reshape(cam.height, cam.width, 3), st


@pytest.fixture(scope="module")
def small_light(device):
    gs = spt.GpuScene(device, scenes.small_light_box_scene().build())
    cam = scenes.box_camera(64, 64)
    ref, _ = _render(gs, cam, scenes.pt_params(spp=16384, path_length=5, seed=99))
    return gs, cam, ref


def _block_means(img, b=8):
    h, w, _ = img.shape
    return img[: h // b * b, : w // b * b].reshape(h // b, b, w // b, b, 3).mean(axis=(1, 3))


def test_guided_render_is_unbiased(device, small_light):
    """On the small-light box guiding does not pay (its light reaches the floor mostly through the halo a
    two-sided emitter makes on the ceiling), but it must stay unbiased: the image mean and every 8 x 8
    block mean agree with a 16,384-spp plain render within their noise, for two independently trained
    guides."""
    gs, cam, ref = small_light
    p = scenes.pt_params(spp=4096, path_length=5, seed=7)
    plain, _ = _render(gs, cam, p)
    bp, br = _block_means(plain), _block_means(ref)
    # the plain render's own block deviations set the noise scale of this comparison
    scale = np.sqrt(np.mean((bp - br) ** 2))
    for seed in (1, 2):
        g = spt.Guide(device, spt.guide_config(batch=1 << 16, max_steps=64, mix=0.5, seed=seed))
        guided, st = _render(gs, cam, p, g)
        assert g.steps > 0
        assert np.isfinite(guided).all()
        assert st.paths == 64 * 64 * 4096
        # the image mean's relative standard error is about 0.35 % at 4096 spp here
        assert abs(float(guided.mean()) - float(ref.mean())) <= 0.015 * float(ref.mean())
        bg = _block_means(guided)
        assert np.sqrt(np.mean((bg - br) ** 2)) < 3.0 * scale + 1e-4, seed
        g.close()


def test_guided_batch_scene_gains(device):
    """A scene of the 64-scene batch set (a dielectric sphere in the lit box, 128 x 128): the trained
    guide lowers the relMSE at an equal sample count and keeps the image mean."""
    sb, _, _, desc = scenes.batched_scenes()[5]
    gs = spt.GpuScene(device, sb.build())
    cam = scenes.box_camera(128, 128)
    ref, _ = _render(gs, cam, scenes.pt_params(spp=16384, path_length=5, seed=99))
    p = scenes.pt_params(spp=1024, path_length=5, seed=7)
    plain, _ = _render(gs, cam, p)
    g = spt.Guide(device, spt.guide_config(batch=1 << 16, max_steps=32, mix=0.5, seed=5))
    guided, _ = _render(gs, cam, p, g)
    g.close()
    assert abs(float(guided.mean()) - float(ref.mean())) <= 0.02 * float(ref.mean())
    e_plain, e_guided = relmse(plain, ref), relmse(guided, ref)
    assert e_guided < 0.8 * e_plain, (desc, e_guided, e_plain)


@pytest.mark.parametrize("idx,seed,depth", [(52, 59, 1), (45, 52, 0)])
def test_guided_batch_scene_stays_finite(device, idx, seed, depth):
    """Two scenes of the 64-scene batch set at their full sizes and 1024 spp: a rough conductor (401 x
    401, 238k triangles) whose training once turned every guide parameter into NaN with this seed, and
    a narrow coated stack (718 x 718) whose guided samples once left NaN pixels.  Both came from the
    vMF sampler's log(0) at a uniform of exactly 0 (one in 2^24) under a narrow lobe."""
    sb, cam, _, desc = scenes.batched_scenes()[idx]
    gs = spt.GpuScene(device, sb.build())
    p = scenes.pt_params(spp=1024, sampler="jittered", termination="max-length", path_length=5, seed=7 + idx)
    plain, _ = _render(gs, cam, p)
    g = spt.Guide(device, spt.guide_config(batch=1 << 18, max_steps=32, mix=0.5, seed=seed, guided_depth=depth))
    guided, _ = _render(gs, cam, p, g)
    grid, mlp = g.get_params()
    g.close()
    assert np.isfinite(grid).all() and np.isfinite(mlp).all(), desc
    assert np.isfinite(guided).all(), (desc, int((~np.isfinite(guided)).sum()))
    assert abs(float(guided.mean()) - float(plain.mean())) <= 0.02 * float(plain.mean()), desc


@pytest.mark.parametrize("mix", [0.5, 0.9])
def test_guided_window_room_is_unbiased_and_less_noisy(device, mix):
    # light enters through a 0.1 x 0.1 window: the sampled lobe and its density (the lobe cache) must
    # agree or the mean drifts, most of all when nearly every direction comes from the guide
    gs = spt.GpuScene(device, scenes.window_room_scene(0.1).build())
    cam = scenes.box_camera(64, 64)
    ref, _ = _render(gs, cam, scenes.pt_params(spp=32768, path_length=5, seed=99))
    p = scenes.pt_params(spp=4096, path_length=5, seed=7)   # 16.8M paths: 25 training steps of 2^16
    plain, _ = _render(gs, cam, p)
    g = spt.Guide(device, spt.guide_config(batch=1 << 16, max_steps=32, mix=mix, seed=1))
    guided, _ = _render(gs, cam, p, g)
    assert np.isfinite(guided).all()
    # the image mean's relative standard error is about 0.2 % at 4096 spp here
    assert abs(float(guided.mean()) - float(ref.mean())) <= 0.02 * float(ref.mean())
    if mix == 0.5:
        e_plain, e_guided = relmse(plain, ref), relmse(guided, ref)
        assert e_guided < 0.8 * e_plain, (e_guided, e_plain)


def test_guided_equals_plain_without_guidable_materials(device):
    # a dielectric over a Lambertian layer: a stack guiding leaves to the reference's walk
    gs = spt.GpuScene(device, scenes.furnace_scene("plastic").build())
    cam = scenes.furnace_camera(32, 32)
    p = scenes.pt_params(spp=16, sampler="regular", termination="russian-roulette", path_length=3, seed=14)
    plain, sp = _render(gs, cam, p)
    g = spt.Guide(device, spt.guide_config(box_min=(-10, -10, -10), box_max=(10, 10, 10), batch=1024, max_steps=4))
    guided, sg = _render(gs, cam, p, g)
    assert sp.segments == sg.segments
    np.testing.assert_allclose(guided, plain, rtol=1e-5, atol=1e-6)


def test_guide_trains_on_its_render(device, small_light):
    gs, cam, _ = small_light
    g = spt.Guide(device, spt.guide_config(batch=1 << 14, max_steps=8, mix=0.5, seed=2))
    grid0, mlp0 = g.get_params()
    _render(gs, cam, scenes.pt_params(spp=64, path_length=5, seed=3), g)
    assert 1 <= g.steps <= 8
    grid1, mlp1 = g.get_params()
    assert not np.array_equal(mlp0, mlp1)
    steps = g.steps
    _render(gs, cam, scenes.pt_params(spp=64, path_length=5, seed=4), g)
    assert steps < g.steps <= steps + 8


def test_guided_coated_material_is_unbiased(device):
    """The 1.3M-triangle scene's material on a smaller mesh: a smooth dielectric (IOR 1.5) over a
    Cook-Torrance layer.  Guiding it mixes the guide with the reference's layered walk through the
    walk's single-internal-bounce component; the rest of the walk keeps its own weight.  Image and
    block means must agree with a plain render within their noise, and with a fully trained guide
    (mix 0.9: nearly every direction from the guide) too."""
    gs = spt.GpuScene(device, scenes.layered_box_scene(4).build())
    cam = scenes.layered_box_camera(64, 48)
    ref, _ = _render(gs, cam, scenes.pt_params(spp=16384, path_length=5, seed=99))
    p = scenes.pt_params(spp=4096, path_length=5, seed=7)
    plain, _ = _render(gs, cam, p)
    br = _block_means(ref)
    scale = np.sqrt(np.mean((_block_means(plain) - br) ** 2))
    for mix in (0.5, 0.9):
        g = spt.Guide(device, spt.guide_config(box_min=(0, 0, 0), box_max=(3, 3, 3), batch=1 << 16,
                                               max_steps=32, mix=mix, seed=3))
        guided, _ = _render(gs, cam, p, g)
        g.close()
        assert np.isfinite(guided).all()
        assert abs(float(guided.mean()) - float(ref.mean())) <= 0.015 * float(ref.mean()), mix
        assert np.sqrt(np.mean((_block_means(guided) - br) ** 2)) < 3.0 * scale + 1e-4, mix
