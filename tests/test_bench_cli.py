"""bench.py's reference arm on CPU: the JSON line the benchmark driver reads (one line, the keys it needs, the
reference's own CPU backend timed with every core, no GPU arm when there is no GPU), the one-line
"unavailable" answer for configurations the reference has no arm for, and a rank other than 0 printing
nothing."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(args, env=None):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                         timeout=300, cwd=ROOT, env={**os.environ, **(env or {})})
    assert out.returncode == 0, out.stderr[-2000:]
    return [line for line in out.stdout.splitlines() if line.strip()]


def test_reference_arm_prints_one_line_with_the_contract_keys():
    import oracle as O
    if not O.reference_available():
        pytest.skip("oracle/_ref is not built here")
    lines = run(["--impl", "reference", "--steps", "1", "--warmup", "0"])
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "images/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "unavailable" in d["reference_cuda"]       # no GPU here


def test_reference_arm_without_a_counterpart_says_why():
    import oracle as O
    if not O.reference_available():
        pytest.skip("oracle/_ref is not built here")
    for config in ("uneven", "differentiable", "mesh_update"):
        (line,) = run(["--impl", "reference", "--config", config, "--steps", "1", "--warmup", "0"])
        d = json.loads(line)
        assert d["impl"] == "reference" and "no reference arm" in d["unavailable"]


def test_reference_arm_on_a_rank_other_than_0_prints_nothing():
    assert run(["--impl", "reference", "--steps", "1", "--warmup", "0"], env={"RANK": "1", "WORLD_SIZE": "2"}) == []
