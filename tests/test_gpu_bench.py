"""The benchmark line's contract on small workloads: `bench.py` prints one
JSON line with the keys the harness reads (value, e2e with its copy
bytes, roofline, clocks, launch count, cpu_baseline / the reference arm's
fields), for the kspn arm and for `--impl reference`."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_kspn_line():
    d = _run("--workload", "rmat20", "--steps", "3", "--warmup", "3", "--no-batched", "--no-other-rmat", "--profile-steps", "0")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "vs_baseline", "dtype", "data",
              "config", "e2e", "gpu_launches", "roofline", "clocks"):
        assert k in d, k
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] >= 3
    assert d["e2e"]["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["achieved"] > 0 and 0 < r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    assert d["gpu_launches"] >= 2 * d["steps"]  # trim_1_first and the resident launch per step
    if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libkspn_ref.so")):
        assert {"value", "unit", "cores", "kind", "sample"} <= set(d["cpu_baseline"])
    assert d["learned_vs_plain"]["workload"]["identical_output"] is True


def test_reference_arm_line():
    d = _run("--impl", "reference", "--workload", "gnm16", "--steps", "2", "--warmup", "1")
    if "unavailable" in d:
        pytest.skip(d["unavailable"])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["config"]["same_graph"] is True
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert {"value", "unit", "cores", "kind", "sample"} <= set(d["cpu_baseline"])
