"""The reference-side binding (include/spt_reference_adapter.hpp) on the GPU: oracle/_ref/adapter_check
(built from the reference's own sources, where they are present, by oracle/Makefile `adapter`) runs
the adapter's GpuRayCaster<DepthRayCaster / NormalRayCaster / IntTestCountRayCaster> and GpuPathTracer
beside the reference's own integrators on one scene: equal ray-caster buffers, statistics and saved
images, and path-traced image means that agree."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "adapter_check")


def test_adapter_integrators_match_reference_integrators(tmp_path):
    if not os.access(EXE, os.X_OK):
        pytest.fail("oracle/_ref/adapter_check is not built: run `make -C oracle adapter` where the reference "
                    "sources are present (build() does)")
    r = subprocess.run([EXE, str(tmp_path)], cwd=str(tmp_path), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "adapter ok" in r.stdout
    for mode in ("depth", "normal", "count"):
        assert (tmp_path / ("gpu_%s.ppm" % mode)).read_bytes() == (tmp_path / ("ref_%s.ppm" % mode)).read_bytes()
