"""B200-native (sm_100a) path-tracing backend with the reference renderer's interfaces.

The CUDA library libspt_cuda.so (built from swpathtracer_b200/csrc) does all ray/scene work; this
package only loads it (native), mirrors its structs (abi), builds scene descriptions and the
synthetic workloads (scenes) and wraps the handles (api).
"""
from . import abi, scenes  # noqa: F401
from .api import (Bvh, Device, GpuScene, Guide, autotune, count_to_rgb_device, default_tune,  # noqa: F401
                  depth_to_rgb_device, guide_config, normal_to_rgb_device, render_batch, rgb_to_bytes_device,
                  write_ppm, write_ppm_bytes)
from .native import SptError  # noqa: F401
