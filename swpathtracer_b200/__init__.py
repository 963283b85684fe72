"""B200-native (sm_100a) path-tracing backend with the reference renderer's interfaces.

The CUDA library libspt_cuda.so (built from swpathtracer_b200/csrc) does all ray/scene work; this
package only loads it (native), mirrors its structs (abi), builds scene descriptions and the
synthetic workloads (scenes) and wraps the handles (api).
"""
from . import abi, scenes  # noqa: F401
from .api import (Bvh, Device, GpuScene, Guide, autotune, default_tune, guide_config, render_batch,  # noqa: F401
                  write_ppm)
from .native import SptError  # noqa: F401
