"""The reference-side binding (include/spt_reference_adapter.hpp) compiles against the reference's own
headers and links with its sources and the product library (oracle/Makefile `adapter`), on the CPU.
Running it on a GPU is tests/test_gpu_adapter.py."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("SPT_REFERENCE_DIR", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "integrators")), reason="reference sources not present")
def test_adapter_builds_against_reference_headers():
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "adapter", "REF=" + REF],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    exe = os.path.join(ROOT, "oracle", "_ref", "adapter_check")
    assert os.access(exe, os.X_OK)
