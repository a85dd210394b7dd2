"""bench.py's reference arm on the host: the JSON line of the CPU oracle on the
single-box workload, and the one-line 'unavailable' answer of the device-only
configurations (ensembles, serving, late-time states)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, timeout=300):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("config", ["c4", "c5", "c6"])
def test_reference_arm_unavailable_for_device_only_configs(config):
    line = run_bench("--config", config, "--impl", "reference")
    assert line["impl"] == "reference" and line["unavailable"]


def test_reference_arm_line_on_the_single_box_workload():
    # configuration 1 (64^3 particles) keeps the CPU suite short; configuration 2 takes
    # the same path with its own state
    line = run_bench("--config", "c1", "--impl", "reference", "--steps", "2", "--warmup", "1")
    assert line["impl"] == "reference"
    assert line["metric"] == "PM step particle-updates/s" and line["unit"] == "particle-updates/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1
    base = line["cpu_baseline"]
    assert base["kind"] == "port" and base["cores"] >= 1 and base["value"] == line["value"]
    assert base["tiles_timed"] == 2 and "tile" in base["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "particle-updates/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["particles"] == 64 ** 3
    assert "int1 x / int2 v" in line["config"]["workload"]
