"""The manifest graph format (kaspan/scc/adapter/manifest.hpp:19-245),
host side: kspn_manifest_write's files are read back by the REFERENCE's own
manifest loader (oracle/_ref) into the same arrays, for every entry width
and both byte orders, and kspn_manifest_read parses the same fields the
reference requires and rejects what it rejects."""
from __future__ import annotations

import os

import numpy as np
import pytest

import kaspan_b200 as K
import oracle as O

WIDTHS = [(8, 4, False), (4, 4, True), (3, 2, False), (8, 8, True), (5, 3, True), (2, 2, False)]


def _graph():
    return O.gnm(300, 1200, 7)


@pytest.mark.parametrize("head_bytes,csr_bytes,big", WIDTHS)
def test_writer_read_by_reference_loader(tmp_path, head_bytes, csr_bytes, big):
    g = _graph()
    if csr_bytes == 1:
        pytest.skip("ids need two bytes here")
    path = K.manifest_write(str(tmp_path), "g", g.n, g.fwh, g.fwc, g.bwh, g.bwc, head_bytes, csr_bytes, big)
    mf = K.manifest_read(path)
    assert (mf.node_count, mf.edge_count, mf.head_bytes, mf.csr_bytes, mf.big_endian) == (g.n, g.m, head_bytes, csr_bytes, int(big))
    assert mf.graph_name == b"g" and mf.schema_version == 1
    assert os.path.getsize(mf.fw_csr_path.decode()) == g.m * csr_bytes
    if O.ref_lib() is None:
        pytest.skip("reference library not built")
    got = O.ref_manifest_load(path)
    assert got is not None
    n, fwh, fwc, bwh, bwc = got
    assert n == g.n
    assert np.array_equal(fwh, g.fwh) and np.array_equal(bwh, g.bwh)
    assert np.array_equal(fwc, g.fwc[: g.m]) and np.array_equal(bwc, g.bwc[: g.m])


def test_byte_order_on_disk(tmp_path):
    g = _graph()
    path = K.manifest_write(str(tmp_path), "b", g.n, g.fwh, g.fwc, g.bwh, g.bwc, 2, 2, True)
    mf = K.manifest_read(path)
    raw = np.fromfile(mf.fw_csr_path.decode(), dtype=">u2")
    assert np.array_equal(raw.astype(np.uint32), g.fwc[: g.m])


def _manifest_text(**over):
    kv = {"schema.version": "1", "graph.code": "x", "graph.name": "x", "graph.endian": "little", "graph.node_count": "3",
          "graph.edge_count": "0", "graph.contains_self_loops": "false", "graph.contains_duplicate_edges": "false",
          "graph.head.bytes": "8", "graph.csr.bytes": "4", "fw.head.path": "a", "fw.csr.path": "b", "bw.head.path": "c", "bw.csr.path": "d"}
    kv.update(over)
    return "% comment\n" + "".join(f"{k} {v}\n" for k, v in kv.items() if v is not None)


@pytest.mark.parametrize("over", [{"graph.endian": "middle"}, {"graph.head.bytes": "9"}, {"graph.csr.bytes": "0"},
                                  {"graph.node_count": "-1"}, {"graph.contains_self_loops": "yes"}, {"bw.csr.path": None}])
def test_parser_rejects(tmp_path, over):
    p = tmp_path / "m.manifest"
    p.write_text(_manifest_text(**over))
    with pytest.raises(K.KspnError):
        K.manifest_read(str(p))


def test_parser_accepts_extra_spaces_and_comments(tmp_path):
    p = tmp_path / "m.manifest"
    p.write_text(_manifest_text().replace("graph.name x", "graph.name    my graph"))
    mf = K.manifest_read(str(p))
    assert mf.graph_name == b"my graph" and mf.node_count == 3
    assert mf.fw_head_path.decode().endswith("/a")
