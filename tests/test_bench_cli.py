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


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_clock_summary_takes_the_samples_of_the_timed_region():
    """nvidia-smi lines (index, clocks.sm, clocks.max.sm, power, active mask, then hw_slowdown,
    hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap): only those from the timed region's start count, or
    the last one before it when the region was shorter than one sampling period."""
    c = _bench().ClockSampler(0)
    c.lines = ["0, 1200, 1965, 300.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1965, 1965, 900.5, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1950, 1965, 950.0, 0x4, Not Active, Not Active, Not Active, Active",
               "garbled"]
    c.start = 1
    assert c.summary() == {"sm_mhz": 1957.5, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 2}
    c.lines = c.lines[:3]
    c.start = 3
    s = c.summary()
    assert s["samples"] == 1 and s["sm_mhz"] == 1950.0
    c.lines, c.start = [], 0
    assert c.summary()["samples"] == 0


def test_algorithmic_bytes_and_profile_figures_the_bench_reports():
    """B_img of the body-worlds image (outputs, inputs and tree build, counted once; 52,068 bytes) and the
    camera kernel's ncu figures the bench line carries, read from the committed profile."""
    import neraulgraphics_b200 as ng
    from neraulgraphics_b200 import workloads
    bench = _bench()
    wl = workloads.body_worlds(worlds=4096, seed=0)
    built = ng.build_meshes(wl.desc.meshes)
    b = bench.algorithmic_bytes_per_image(wl, built["nodes"].nbytes + built["triangles"].nbytes)
    assert round(b) == 52068
    assert 64 * 64 * 11 < b < 64 * 64 * 11 + 8000
    traffic = bench.traffic_per_image()
    assert traffic is not None and 45056 <= traffic < 1e6
    f = bench.issue_figures()
    assert 0 < f["threads_per_warp_instruction"] <= 32 and 0 < f["issue_active_pct"] <= 100
    assert 0 < f["warps_active_pct"] <= 100
