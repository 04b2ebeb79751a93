"""``bench.py`` keeps its output contract on a GPU: one JSON line with the
metric, the device-resident value, the end-to-end value with its copied
bytes, the roofline of the dominant kernel, the sampled clocks and the
count of this library's kernel launches."""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_headline_line_has_every_contract_key(require_gpu):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "1",
                          "--warmup", "3", "--no-cpu", "--no-public",
                          "--no-serving"], capture_output=True,
                         text=True,
                         cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "e2e",
              "roofline", "clocks", "gpu_launches"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 3
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "uneven_batch_256"
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert 0 < r["frac"] < 1.5 and r["achieved"] > 0 and r["peak"] > 0
    assert r["traffic"] > 0 and r["kernel"] == "engine_persistent"
    assert d["gpu_launches"] > 0
    assert "sm_mhz" in d["clocks"]
    # the plain one-LP-at-a-time arm on the same mix, and the latency percentiles
    one = d["one_at_a_time"]
    assert one["value"] > 0 and d["vs_baseline"] == pytest.approx(e["value"] / one["value"])
    for lat in (d["latency_s"], one["latency_s"], one["service_s"]):
        assert 0 < lat["p50"] <= lat["p99"]
