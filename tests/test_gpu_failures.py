"""The failure statuses the wavefront writes, made to fire from the host and checked on the GPU.

Nothing here faults, traps or hangs the device: the iteration budget is a host-set limit that the
render loop's own continuation kernel checks (k_continue sets the timeout bit and ends the loop), and
the stack limit makes the traversal set the overflow bit instead of pushing.  After each failure the
same context renders again and must give the same image as a clean render.
"""
import numpy as np
import pytest
import torch

import swpathtracer_b200 as spt
from swpathtracer_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu


def _render(device, gs, cam, params, tune=None):
    buf = torch.zeros(cam.width * cam.height * 3, dtype=torch.float32, device="cuda")
    st = spt.render_batch(device, [(gs, cam, params)], [buf.data_ptr()], tune=tune)
    torch.cuda.synchronize()
    return buf.cpu().numpy().reshape(cam.height, cam.width, 3), st[0]


@pytest.fixture(scope="module")
def box(device):
    gs = spt.GpuScene(device, scenes.box_scene(3).build())
    yield gs
    gs.close()


def test_iteration_budget_ends_the_render_with_timeout(device, box):
    cam = scenes.box_camera(64, 48)
    p = scenes.pt_params(spp=16, termination="max-length", path_length=5, seed=9)
    clean, _ = _render(device, box, cam, p)
    t = spt.default_tune()
    t.max_iterations = 1
    with pytest.raises(native.SptError) as e:
        _render(device, box, cam, p, t)
    assert e.value.status == abi.SPT_ERR_TIMEOUT
    # the context is usable afterwards, and a budget that suffices changes nothing
    again, _ = _render(device, box, cam, p)
    assert np.allclose(again, clean, rtol=1e-5, atol=1e-6)
    t.max_iterations = 100000
    enough, _ = _render(device, box, cam, p, t)
    assert np.allclose(enough, clean, rtol=1e-5, atol=1e-6)


def test_stack_limit_overflow_is_reported(device):
    gs = spt.GpuScene(device, scenes.displaced_mesh_scene(6).build())
    cam = scenes.displaced_mesh_camera(96, 54)
    p = scenes.pt_params(spp=4, termination="max-length", path_length=3, seed=5)
    clean, _ = _render(device, gs, cam, p)
    t = spt.default_tune()
    t.stack_limit = 1
    with pytest.raises(native.SptError) as e:
        _render(device, gs, cam, p, t)
    assert e.value.status == abi.SPT_ERR_OVERFLOW
    again, _ = _render(device, gs, cam, p)
    assert np.allclose(again, clean, rtol=1e-5, atol=1e-6)
    # every compiled stack depth that holds the tree gives the same image
    for depth in (16, 24, 32):
        t = spt.default_tune()
        t.stack = depth
        img, _ = _render(device, gs, cam, p, t)
        assert np.allclose(img, clean, rtol=1e-5, atol=1e-6), depth
    gs.close()


def test_bad_tune_values_are_rejected(device, box):
    cam = scenes.box_camera(16, 16)
    p = scenes.pt_params(spp=1, seed=1)
    for field, value in (("stack", 20), ("shade_block", 48), ("traversal", 5)):
        t = spt.default_tune()
        setattr(t, field, value)
        with pytest.raises(native.SptError) as e:
            _render(device, box, cam, p, t)
        assert e.value.status == abi.SPT_ERR_INVALID_ARGUMENT, field
