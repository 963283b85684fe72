"""The ray casters' post-processing and the PPM quantization on the GPU against the oracle's restatement
of integrators/depth_raycaster.cpp:9-34, int_test_count_raycaster.cpp:20-73 and core/image_buffer.cpp:22-47."""
import numpy as np
import pytest
import torch

import swpathtracer_b200 as spt
from swpathtracer_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _raycast(device, mode):
    gs = spt.GpuScene(device, scenes.box_scene(4).build())
    cam = scenes.box_camera(96, 72)
    img, st = gs.raycast(cam, mode, stats=True)
    return img, st, cam


@pytest.mark.parametrize("prescribed", [(-1.0, -1.0), (0.5, 3.0)])
def test_depth_ramp_matches_oracle(device, oracle, prescribed):
    depth, _, cam = _raycast(device, abi.RAYCAST_DEPTH)
    d_in = torch.from_numpy(depth.astype(np.float32)).cuda()
    d_out = torch.empty((cam.height, cam.width, 3), dtype=torch.float32, device="cuda")
    spt.depth_to_rgb_device(device, d_in.data_ptr(), cam.width, cam.height, d_out.data_ptr(), *prescribed)
    torch.cuda.synchronize()
    exp = oracle.depth_to_rgb(depth, *prescribed)
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32), exp.view(np.uint32))


@pytest.mark.parametrize("prescribed", [(-1, -1), (10, 200)])
def test_count_heat_map_matches_oracle(device, oracle, prescribed):
    count, st, cam = _raycast(device, abi.RAYCAST_COUNT)
    d_in = torch.from_numpy(count.astype(np.int64)).cuda()
    d_out = torch.empty((cam.height, cam.width, 3), dtype=torch.float32, device="cuda")
    spt.count_to_rgb_device(device, d_in.data_ptr(), cam.width, cam.height, d_out.data_ptr(), *prescribed)
    torch.cuda.synchronize()
    exp = oracle.count_to_rgb(count, st.min_tests_pp, st.max_tests_pp, *prescribed)
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32), exp.view(np.uint32))


def test_bytes_and_ppm_match_the_host_writer(device, tmp_path):
    rng = np.random.default_rng(4)
    rgb = np.concatenate([rng.uniform(-0.2, 1.3, 30000), np.linspace(0, 1, 3001)]).astype(np.float32)
    rgb = rgb[: (len(rgb) // 3) * 3].reshape(1, -1, 3)
    d_in = torch.from_numpy(rgb).cuda()
    d_out = torch.empty(rgb.size, dtype=torch.uint8, device="cuda")
    for srgb in (True, False):
        spt.rgb_to_bytes_device(device, d_in.data_ptr(), rgb.size, d_out.data_ptr(), srgb=srgb)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        spt.write_ppm(str(tmp_path / "host.ppm"), rgb, srgb=srgb)
        host = np.array([int(v) for v in (tmp_path / "host.ppm").read_text().split()[4:]], np.int64)
        diff = np.abs(got.astype(np.int64) - host)
        assert diff.max() <= 1 and (diff == 0).mean() > 0.9999
        spt.write_ppm_bytes(str(tmp_path / "dev.ppm"), got.reshape(rgb.shape))
        if diff.max() == 0:
            assert (tmp_path / "dev.ppm").read_text() == (tmp_path / "host.ppm").read_text()
