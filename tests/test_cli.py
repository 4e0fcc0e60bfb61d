"""kspn_bench, the bench_kaspan command line (tool/bench_kaspan/src/main.cpp)
on the GPU: the reference's arguments, its statistic JSON layout
(kaspan/debug/statistic.hpp:123-205), and the component count it reports
equal to the oracle Tarjan's on the same seeded graph."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

import kaspan_b200 as K
import oracle as O

CLI = os.path.join(os.path.dirname(K.__file__), "kspn_bench")


def test_usage_without_arguments():
    if not os.path.exists(CLI):
        pytest.skip("kspn_bench not built")
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode == 1 and "usage:" in r.stderr


def _run(tmp_path, *args):
    out = tmp_path / "stats.json"
    r = subprocess.run([CLI, *args, "--output_file", str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(out.read_text())["0"]["benchmark"]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [None, "fast", "trim_ex_residual"])
def test_kagen_gnm(tmp_path, variant):
    args = ["--kagen_option_string", "gnm-directed;n=65536;m=524288;seed=1"] + (["--variant", variant] if variant else [])
    b = _run(tmp_path, *args)
    g = O.gnm(65536, 524288, 1)
    assert b["n"] == g.n and b["m"] == g.m and b["world_size"] == 1
    assert b["global_component_count"] == len(np.unique(O.tarjan(g)))
    assert "trim_1_first" in b["scc"] and b["scc"]["trim_1_first"]["decided_count"] > 0
    assert sum(v["decided_count"] for v in b["scc"].values() if isinstance(v, dict)) == g.n
    assert b["kagen"]["duration"] > 0 and b["scc"]["duration"] > 0


@pytest.mark.gpu
def test_kagen_rmat_and_manifest(tmp_path):
    b = _run(tmp_path, "--kagen_option_string", "rmat;directed;n=4096;m=65536;a=0.57;b=0.19;c=0.19;seed=3")
    g = O.rmat(12, 16, 3)
    assert b["m"] == g.m and b["global_component_count"] == len(np.unique(O.tarjan(g)))
    path = K.manifest_write(str(tmp_path), "r", g.n, g.fwh, g.fwc, g.bwh, g.bwc, 4, 3, True)
    b2 = _run(tmp_path, "--manifest_file", path, "--variant", "fast")
    assert b2["m"] == g.m and b2["global_component_count"] == b["global_component_count"]
    assert b2["load"]["duration"] > 0
