"""bench.py on the CPU: the reference arm's JSON line and the CPU baselines.

The reference arm (``--impl reference``) runs the reference evolver built from
its own sources (oracle/_ref/ref32) on the host cores, so its contract can be
checked without a GPU: one JSON line with ``impl: reference``, the metric and
unit of the GPU arm, a ``cpu_baseline`` describing the run and an ``e2e`` with
no host-device traffic.  The FP64 baseline (oracle/_ref/ref64) is the figure
reported beside the FP64 form.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import refrun  # noqa: E402


def _need_reference(fp64=False):
    if not refrun.available(fp64):
        pytest.skip("oracle/_ref not built (needs the reference sources)")


def test_reference_arm_json_line():
    _need_reference()
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "site-updates/s" and d["unit"] == "site-updates/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and "ref32" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


@pytest.mark.parametrize("fp64", [False, True])
def test_cpu_reference_throughput(fp64):
    _need_reference(fp64)
    import bench
    r = bench.cpu_reference_throughput("sm", 12, 2, 2, fp64=fp64)
    assert r["kind"] == "reference" and r["cores"] == 2 and r["value"] > 0 and r["per_process"] > 0
    assert ("ref64" if fp64 else "ref32") in r["sample"]
