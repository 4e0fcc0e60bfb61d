"""CPU: the C-ABI library loads, exports every entry point include/kspn.h
declares, and its host-side logic answers without a GPU."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

import kaspan_b200 as K

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "kspn.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kspn_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ("kspn_scc", "kspn_scc_device", "kspn_strerror", "kspn_trim_1_first", "kspn_forward_backward_search",
              "kspn_trim_1_normal", "kspn_label_search", "kspn_trim_1_exhaustive_first", "kspn_normalise", "kspn_transpose"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    L = K.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    # and the Python bindings cover the whole header
    assert set(declared_symbols()) <= set(K.SIGNATURES)


def test_struct_layouts_match_header():
    # struct_size is what the library itself reports for kspn_options
    o = K.Options()
    assert K.lib().kspn_options_default(C.byref(o)) == 0
    assert o.struct_size == C.sizeof(K.Options)
    assert K.lib().kspn_options_size() == C.sizeof(K.Options)
    assert K.lib().kspn_stats_size() == C.sizeof(K.Stats)
    assert o.pipeline == K.PIPELINE_FAST and o.trim2 == 1 and o.validate == 1


def test_strerror_covers_every_status():
    L = K.lib()
    for code in range(8):
        assert L.kspn_strerror(code)
    assert L.kspn_strerror(99) == b"unknown status"


def test_no_device_is_an_error_not_a_crash():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert K.lib().kspn_context_create(0, C.byref(h)) == 6  # KSPN_ERR_NO_DEVICE
    assert K.lib().kspn_context_create(-1, C.byref(h)) == 6
    assert K.lib().kspn_context_create(0, None) == 1
    with pytest.raises(K.KspnError):
        K.Context(0)


def test_null_context_is_rejected():
    L = K.lib()
    assert L.kspn_scc_device(None, 1, 0, None, None, None, None, None, None, None) == 1
    assert L.kspn_normalise(None, 1, None) == 1
    assert L.kspn_options_default(None) == 1


STANDIN_VIEW = r"""
#include <kaspan_b200/scc.hpp>
#include <cstdint>
// the members of the reference's bidi_graph_part_view<single_part_view>
// (kaspan/graph/bidi_graph_part.hpp:12-28) with index_t = INDEX
struct part_t { std::uint32_t n_; std::uint32_t n() const { return n_; } int world_size() const { return 1; } };
struct view { part_t part; INDEX local_fw_m, local_bw_m; struct { INDEX* head; std::uint32_t* csr; } fw, bw; };
void call(view v, std::uint32_t* ids) { kaspan_b200::scc(v, ids); }
"""


@pytest.mark.parametrize("index", ["std::uint64_t", "std::uint32_t"])
def test_cpp_dropin_header_compiles(tmp_path, index):
    """The C++ drop-in instantiates for 64- and 32-bit offsets (the 32-bit
    path widens them on the host) against a stand-in with the reference
    view's members; the GPU test runs it on the reference's own type."""
    import shutil
    import subprocess

    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    src = tmp_path / "standin.cpp"
    src.write_text(STANDIN_VIEW)
    inc = os.path.join(os.path.dirname(HEADER))
    r = subprocess.run([gxx, "-std=c++20", "-fsyntax-only", f"-DINDEX={index}", "-I", inc, str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
