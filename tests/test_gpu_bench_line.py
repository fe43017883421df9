"""The benchmark's JSON line on a small case: one line on stdout with the keys and units the
measurement contract needs (throughput, end-to-end figure with its host<->device bytes, the
dominant kernel's roofline, per-kernel figures, clocks, launch count), all finite."""
import json
import math
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_bench_line_fields_small_case():
    d = _run("--config", "rbc3d_small", "--steps", "3", "--warmup", "3", "--no-cpu-baseline")
    assert d["metric"] == "Mcell-RK3-steps/s" and d["unit"] == "Mcell-RK3-steps/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3
    assert d["value"] > 0 and math.isfinite(d["value"]) and d["ms_per_step"] > 0
    assert d["dtype"] == "f64" and d["config"]["workload"] == "rbc3d_128x128x256_fp64_ra1e9"
    e = d["e2e"]
    assert 0 < e["value"] <= d["value"] * 1.05 and e["unit"] == d["unit"]
    nx, ny, nz = 257, 128, 128
    assert e["h2d_bytes_per_step"] == 5 * nx * ny * nz * 8 // 3
    assert e["d2h_bytes_per_step"] >= e["h2d_bytes_per_step"]
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["kernel"] == "k_explicit_implicit"
    assert 0 < r["frac"] < 1.5 and r["peak"] > 0
    assert r["algorithmic_bytes_per_launch"] == 136 * 256 * 128 * 128
    kr = d["kernels_roofline"]
    for k in ("explicit_implicit", "div_fft_y", "fft_z_fwd", "tridiag_pressure", "fft_z_inv", "ifft_y", "correct"):
        assert 0 < kr[k]["frac"] < 1.5 and kr[k]["ms_per_launch"] > 0, k
    assert d["gpu_launches"] > 0
    assert "sm_mhz" in (d["clocks"] or {"sm_mhz": None})
    assert d["vs_baseline"] is None
