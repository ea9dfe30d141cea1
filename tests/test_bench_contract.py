"""The reference arm of bench.py on the CPU: one JSON line with the keys the
benchmark contract needs (metric, value, unit, impl, cpu_baseline, e2e), for a
3D, the 2D and the mask-builder workload.  The arm times the reference's own CPU solver built from
its sources (oracle/_ref); without that build the test is skipped."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF3D = os.path.join(ROOT, "oracle", "_ref", "libref3d.so")
REF2D = os.path.join(ROOT, "oracle", "_ref", "libref2d.so")


def _reference_line(config: str) -> dict:
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", config,
                          "--steps", "1", "--warmup", "0", "--ref-budget", "30"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


@pytest.mark.parametrize("config,lib", [("spheres64", REF3D), ("channel2d", REF2D)])
def test_reference_arm_json(config, lib):
    if not os.path.exists(lib):
        pytest.skip("the reference build (oracle/_ref) is not present")
    d = _reference_line(config)
    assert d["impl"] == "reference"
    assert d["metric"] == "cell-steps/s" and d["unit"] == "cell-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] >= 1
    assert d["config"]["workload"].startswith(config)
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_json_masks():
    """The mask-builder workload's reference arm: the reference's own Grid3D::Prepare,
    timed in cells per second."""
    if not os.path.exists(REF3D):
        pytest.skip("the reference build (oracle/_ref) is not present")
    d = _reference_line("masks262")
    assert d["impl"] == "reference" and d["metric"] == "cells/s" and d["unit"] == "cells/s"
    assert d["value"] > 0 and d["steps"] >= 1 and d["config"]["cells"] == 262 * 262 * 264
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"]
