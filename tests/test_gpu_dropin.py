"""GPU: the C++ drop-in include/kaspan_b200/scc.hpp against the reference's
own view type and entry point.  oracle/_ref/dropin_check64 and
dropin_check32 (built from oracle/dropin_check.cpp with the reference's
headers, with and without KASPAN_INDEX64) pass one
bidi_graph_part_view<single_part_view> to kaspan::scc + normalise_scc_id
(kaspan/scc/scc.hpp:21-25, kaspan/test/normalise_scc.hpp:10-25) and to
kaspan_b200::scc, and exit 0 when every graph gives the same ids; the u32
build runs the drop-in's host-side widening of 32-bit offsets."""
from __future__ import annotations

import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("index_bits", [64, 32])
def test_cpp_dropin_matches_reference(index_bits):
    exe = os.path.join(ROOT, "oracle", "_ref", f"dropin_check{index_bits}")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref drop-in check not built (reference sources absent at build time)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dropin check ok" in r.stdout
    assert "DIFFERENT" not in r.stdout
