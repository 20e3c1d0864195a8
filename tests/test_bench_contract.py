"""bench.py's one-line JSON contract, on small cases: the reference arm on
the host (CPU) and this repository's arm on the GPU."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, timeout=900):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


def check_common(d):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config"):
        assert k in d, k
    assert d["value"] > 0 and d["unit"] == "Mrays/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["scaling"] == "weak" and "workload" in d["config"]
    c = d["config"]
    assert c["resolution"] == [1920, 1080] and c["spp"] == 64 and c["technique"] == "pt.mis"
    assert c["max_path_vertices"] == 17 and c["rr_depth"] == 5 and c["triangles"] == 3404098


@pytest.mark.skipif(not oracle.ref_available("f"), reason="reference tree not present: harness not built")
def test_reference_arm_line():
    d = run_bench("--impl", "reference", "--steps", "1", "--warmup", "1")
    check_common(d)
    assert d["impl"] == "reference"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # The reference traces a shadow ray at every non-delta vertex, whatever
    # the light sample contributes: about five rays per sample on this scene.
    assert 3.0 < d["rays_per_sample"] < 8.0


@pytest.mark.gpu
def test_gpu_arm_line(cuda):
    # One sample per pixel per frame keeps the test short; the line's shape
    # is the full run's.
    d = run_bench("--steps", "3", "--warmup", "3", "--render-spp", "1", "--sections=", "--no-cpu-baseline",
                  "--no-render-parity", "--no-autotune")
    check_common(d)
    assert "impl" not in d or d["impl"] != "reference"
    assert d["steps"] == 3 and d["warmup"] == 3 and d["gpu_launches"] >= 3
    r = d["roofline"]
    assert r["unit"] == "GB/s" and 0 < r["frac"] < 2 and r["peak"] > 0
    assert abs(r["achieved"] / r["peak"] - r["frac"]) < 1e-3
    assert r["kernels"]["closest"]["node_tests_per_ray"] > 1 and r["kernels"]["shadow"]["rays"] > 0
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] == 1920 * 1080 * 3 * 4
    assert set(d["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    assert 1.0 < d["rays_per_sample"] < 8.0
