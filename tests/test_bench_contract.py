"""bench.py --impl reference on the CPU: one JSON line on the GPU arm's metric, unit and workload.

The reference arm times the reference's own closest-hit traversal (oracle/_ref, or the oracle's
restatement when the reference was not built) on the host cores, on a bounded sample of the
headline workload.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


@pytest.fixture(scope="module")
def reference_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-3000:]
    return json.loads(lines[0])


def test_reference_arm_reports_the_headline_metric(reference_line):
    d = reference_line
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "Mrays/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == bench.WORKLOAD
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1


def test_reference_arm_describes_its_cpu_baseline(reference_line):
    d = reference_line
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_profile_commands_use_flags_bench_accepts():
    """Every `python bench.py ...` command quoted in profiles/ parses with bench.py's own argument
    parser, so a profile's recipe keeps running the committed bench as it stands."""
    import glob
    import re
    import shlex
    cmds = []
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        text = open(path).read().replace("\\\n", " ")
        for m in re.finditer(r"python bench\.py([^\n>|&`]*)", text):
            cmds.append((os.path.basename(path), shlex.split(m.group(1))))
    assert cmds, "no bench commands found in profiles/"
    for name, argv in cmds:
        old = sys.argv
        try:
            sys.argv = ["bench.py"] + argv
            bench.args_()
        except SystemExit as e:
            pytest.fail("%s: bench.py rejects %s (%s)" % (name, argv, e))
        finally:
            sys.argv = old
