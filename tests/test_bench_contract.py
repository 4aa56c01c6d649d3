"""bench.py's reference arm on the host: one JSON line with the GPU arm's
metric, unit and `config` object (identical keys and values, so the two lines
compare), the CPU it ran on, and an end-to-end entry with no device copies."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_line_matches_the_gpu_arm_contract():
    sys.path.insert(0, str(ROOT))
    import bench
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["config"] == json.loads(json.dumps(bench.WORKLOAD))
    assert line["config"]["workload"].startswith("nside1024_")
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["nproc"] >= 1 and cb["cpu_model"]
    assert cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_cpu_sample_is_proportional_to_the_day():
    """The sample takes the same fraction of the day's half-baselines and
    pixels, so its term mix is the day's."""
    sys.path.insert(0, str(ROOT))
    import bench
    inp = bench.cpu_inputs()
    s1, s2 = bench.cpu_sample_sizes(inp, 0.5)
    f1, f2 = s1 / inp["n_half"], s2 / inp["npix"]
    assert 0 < f1 < 1 and abs(f1 - f2) <= max(f1, f2) * 0.05 + 16 / inp["n_half"]
