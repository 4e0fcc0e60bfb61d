"""CPU checker for the kspn CUDA library -- TEST INFRASTRUCTURE ONLY.

Python access (ctypes + numpy) to two CPU libraries built by oracle/Makefile:

* ``libkspn_oracle.so`` -- the plain-C restatement of the reference's
  single-rank SCC path (oracle/kspn_oracle.c; every function there cites the
  rawbby/KaSpan file:line it follows) plus the CPU side of the seeded graph
  generators;
* ``_ref/libkspn_ref.so`` -- the reference's own code, compiled from its
  sources as one rank (oracle/ref_bridge.cpp).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference leg import this module.  The product (kaspan_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
UNDECIDED = 0xFFFFFFFF

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

_orc = None
_ref = None


def build() -> None:
    """Build both checker libraries (the reference one only where its sources exist)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _orc
    if _orc is None:
        path = os.path.join(HERE, "libkspn_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        u32, u64, i32, dbl = C.c_uint32, C.c_uint64, C.c_int, C.c_double
        sig = {
            "orc_normalise": (None, [u32, _u32p]),
            "orc_tarjan": (u32, [u32, _u64p, _u32p, _u32p]),
            "orc_trim_1_first": (u32, [u32, _u64p, _u64p, _u8p, _u32p, C.c_void_p]),
            "orc_trim_1_normal": (u32, [u32, _u64p, _u32p, _u64p, _u32p, _u8p, _u32p]),
            "orc_fw_bw": (u32, [u32, _u64p, _u32p, _u64p, _u32p, _u8p, _u32p, u32]),
            "orc_label_search_pull": (u32, [u32, _u64p, _u32p, _u64p, _u32p, _u8p, _u32p, i32, C.c_void_p]),
            "orc_trim_1_exhaustive_first": (u32, [u32, u64, _u64p, _u32p, _u64p, _u32p, _u8p, _u32p, _u32p, _u32p]),
            "orc_trim_1_fixpoint": (u32, [u32, _u64p, _u32p, _u64p, _u32p, _u8p, _u32p]),
            "orc_scc": (u32, [u32, _u64p, _u32p, _u64p, _u32p, _u32p, C.c_void_p]),
            "orc_seed_key": (u64, [u64]),
            "orc_draw": (u64, [u64, u64]),
            "orc_gen_gnm": (None, [u32, u64, u64, _u32p, _u32p]),
            "orc_rmat_perm": (u32, [u32, i32, u64]),
            "orc_gen_rmat": (None, [i32, u64, u64, u64, u64, u64, i32, _u32p, _u32p]),
            "orc_rgg_points": (None, [u32, u64, u32, _u32p, _u32p, _u64p]),
            "orc_rgg_edges": (u64, [u32, u64, u32, u64, _u32p, _u32p, _u64p, _u64p, C.c_void_p, C.c_void_p]),
            "orc_build_csr": (u64, [u32, u64, _u32p, _u32p, _u64p, _u32p]),
            "orc_transpose": (None, [u32, _u64p, _u32p, _u64p, _u32p]),
            "orc_fuzzy": (u64, [u64, u32, dbl, _u32p, _u64p, _u32p, u64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _orc = L
    return _orc


def ref_lib() -> C.CDLL | None:
    """The reference's own code (None when oracle/_ref was never built)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libkspn_ref.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        u32, u64, i32, i64 = C.c_uint32, C.c_uint64, C.c_int, C.c_int64
        sig = {
            "kref_scc": (i64, [i32, u32, u64, _u64p, _u32p, _u64p, _u32p, _u32p]),
            "kref_tarjan": (i64, [u32, u64, _u64p, _u32p, _u32p]),
            "kref_normalise": (None, [u32, _u32p]),
            "kref_trim_1_first": (u32, [u32, u64, _u64p, _u32p, _u64p, _u32p, _u64p, _u32p]),
            "kref_fw_bw": (None, [u32, u64, _u64p, _u32p, _u64p, _u32p, _u64p, _u32p, u32]),
            "kref_trim_1_normal": (None, [u32, u64, _u64p, _u32p, _u64p, _u32p, _u64p, _u32p]),
            "kref_label_search_pull": (None, [u32, u64, _u64p, _u32p, _u64p, _u32p, _u64p, _u32p, i32]),
            "kref_trim_1_exhaustive_first": (None, [u32, u64, _u64p, _u32p, _u64p, _u32p, _u64p, _u32p, _u32p, _u32p]),
            "kref_select_pivot_from_degree": (u32, [u32, _u64p, _u32p, _u32p]),
            "kref_manifest_load": (i32, [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _ref = L
    return _ref


# --------------------------------------------------------------------------
# graphs
# --------------------------------------------------------------------------
@dataclass
class Graph:
    n: int
    fwh: np.ndarray  # uint64[n+1]
    fwc: np.ndarray  # uint32[m]
    bwh: np.ndarray  # uint64[n+1]
    bwc: np.ndarray  # uint32[m]

    @property
    def m(self) -> int:
        return int(self.fwh[-1]) if self.n else 0


def _arr32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a if a.size else np.zeros(1, np.uint32)


def from_csr(n: int, fwh, fwc) -> Graph:
    fwh = np.ascontiguousarray(fwh, dtype=np.uint64)
    fwc = _arr32(fwc)
    bwh, bwc = transpose(n, fwh, fwc)
    return Graph(n, fwh, fwc, bwh, bwc)


def transpose(n, fwh, fwc):
    m = int(fwh[-1]) if n else 0
    bwh = np.zeros(n + 1, np.uint64)
    bwc = np.zeros(max(m, 1), np.uint32)
    lib().orc_transpose(n, fwh, fwc, bwh, bwc)
    return bwh, bwc


def from_edges(n: int, src, dst) -> Graph:
    """Self-loops and duplicates removed, rows ascending (orc_build_csr)."""
    src = _arr32(src)
    dst = _arr32(dst)
    m_raw = int(np.asarray(src).size)
    fwh = np.zeros(n + 1, np.uint64)
    fwc = np.zeros(max(m_raw, 1), np.uint32)
    m = lib().orc_build_csr(n, m_raw, src, dst, fwh, fwc)
    return from_csr(n, fwh, fwc[: max(m, 1)].copy() if m else np.zeros(1, np.uint32))


def gnm_edges(n: int, draws: int, seed: int):
    src = np.empty(max(draws, 1), np.uint32)
    dst = np.empty(max(draws, 1), np.uint32)
    lib().orc_gen_gnm(n, draws, seed, src, dst)
    return src[:draws], dst[:draws]


def gnm(n: int, draws: int, seed: int) -> Graph:
    return from_edges(n, *gnm_edges(n, draws, seed))


def rmat_thresholds(a: float, b: float, c: float):
    s = float(1 << 32)
    return int(math.floor(a * s)), int(math.floor((a + b) * s)), int(math.floor((a + b + c) * s))


def rmat_edges(scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19, permute=True):
    draws = edge_factor << scale
    ta, tab, tabc = rmat_thresholds(a, b, c)
    src = np.empty(max(draws, 1), np.uint32)
    dst = np.empty(max(draws, 1), np.uint32)
    lib().orc_gen_rmat(scale, draws, seed, ta, tab, tabc, 1 if permute else 0, src, dst)
    return src[:draws], dst[:draws]


def rmat(scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19, permute=True) -> Graph:
    return from_edges(1 << scale, *rmat_edges(scale, edge_factor, seed, a, b, c, permute))


def rgg_params(n: int, mean_undirected_degree: float = 8.0):
    """Radius for the requested mean degree (boundary effects ignored), the
    cell count per side g = floor(1/r) and r^2 in 2^-60 fixed point."""
    r2 = mean_undirected_degree / (math.pi * n)
    r = math.sqrt(r2)
    g = max(1, int(math.floor(1.0 / r)))
    r2_fixed = int(math.floor(r2 * float(1 << 60)))
    return g, r2_fixed


def rgg(n: int, seed: int, mean_undirected_degree: float = 8.0) -> Graph:
    g, r2 = rgg_params(n, mean_undirected_degree)
    L = lib()
    px = np.empty(max(n, 1), np.uint32)
    py = np.empty(max(n, 1), np.uint32)
    cs = np.empty(g * g + 1, np.uint64)
    L.orc_rgg_points(n, seed, g, px, py, cs)
    off = np.zeros(n + 1, np.uint64)
    m = L.orc_rgg_edges(n, seed, g, r2, px, py, cs, off, None, None)
    src = np.empty(max(m, 1), np.uint32)
    dst = np.empty(max(m, 1), np.uint32)
    L.orc_rgg_edges(n, seed, g, r2, px, py, cs, off, src.ctypes.data, dst.ctypes.data)
    return from_edges(n, src[:m], dst[:m])


def fuzzy(seed: int, n: int, d: float = -1.0):
    """Planted-partition graph (oracle/kspn_oracle.c orc_fuzzy); returns
    (graph, planted min-id labels)."""
    cap = max(16, int(max(d, 0) * n) + 2 * n + 16) if d != -1.0 else max(16, n * n)
    scc_id = np.zeros(max(n, 1), np.uint32)
    fwh = np.zeros(n + 1, np.uint64)
    fwc = np.zeros(max(cap, 1), np.uint32)
    m = lib().orc_fuzzy(seed, n, d, scc_id, fwh, fwc, cap)
    g = from_csr(n, fwh, fwc[: max(m, 1)].copy())
    return g, scc_id[:n].copy()


# --------------------------------------------------------------------------
# algorithms (restatement)
# --------------------------------------------------------------------------
def tarjan(g: Graph) -> np.ndarray:
    out = np.zeros(max(g.n, 1), np.uint32)
    lib().orc_tarjan(g.n, g.fwh, g.fwc, out)
    return out[: g.n]


def normalise(ids: np.ndarray) -> np.ndarray:
    ids = np.ascontiguousarray(ids, dtype=np.uint32).copy()
    if ids.size:
        lib().orc_normalise(ids.size, ids)
    return ids


def scc(g: Graph):
    """Default pipeline restated; returns (normalised ids, per-phase decided, label calls)."""
    out = np.zeros(max(g.n, 1), np.uint32)
    pd = np.zeros(4, np.uint32)
    calls = lib().orc_scc(g.n, g.fwh, g.fwc, g.bwh, g.bwc, out, pd.ctypes.data)
    return normalise(out[: g.n]), pd, calls


def new_state(n: int):
    return np.ones(max(n, 1), np.uint8), np.full(max(n, 1), UNDECIDED, np.uint32)


def bits_from_bytes(und: np.ndarray, n: int) -> np.ndarray:
    words = np.zeros((n + 63) // 64 or 1, np.uint64)
    idx = np.nonzero(und[:n])[0]
    np.bitwise_or.at(words, idx // 64, (np.uint64(1) << (idx % 64).astype(np.uint64)))
    return words


def bytes_from_bits(words: np.ndarray, n: int) -> np.ndarray:
    k = np.arange(n)
    return ((words[k // 64] >> (k % 64).astype(np.uint64)) & np.uint64(1)).astype(np.uint8)


# --------------------------------------------------------------------------
# the reference itself (compiled from its sources)
# --------------------------------------------------------------------------
VARIANTS = {
    "scc": 0,
    "hpc_like": 1,
    "hpc_trim_ex": 2,
    "ispan_like": 3,
    "trim_ex": 4,
    "trim_ex_light_residual": 5,
    "trim_ex_residual": 6,
}


def ref_scc(g: Graph, variant: str = "scc"):
    """Reference kaspan::scc (or a variant); returns (normalised ids, seconds)."""
    R = ref_lib()
    out = np.zeros(max(g.n, 1), np.uint32)
    ns = R.kref_scc(VARIANTS[variant], g.n, g.m, g.fwh, g.fwc, g.bwh, g.bwc, out)
    ids = out[: g.n].copy()
    if g.n:
        R.kref_normalise(g.n, ids)
    return ids, ns * 1e-9


def ref_manifest_load(path: str):
    """The reference's manifest loader on `path`: (n, fwh, fwc, bwh, bwc) or None."""
    R = ref_lib()
    n, m = C.c_uint64(), C.c_uint64()
    if R.kref_manifest_load(path.encode(), C.byref(n), C.byref(m), None, None, None, None) != 0:
        return None
    fwh = np.zeros(n.value + 1, np.uint64)
    bwh = np.zeros(n.value + 1, np.uint64)
    fwc = np.zeros(max(m.value, 1), np.uint32)
    bwc = np.zeros(max(m.value, 1), np.uint32)
    if R.kref_manifest_load(path.encode(), C.byref(n), C.byref(m), fwh.ctypes.data, fwc.ctypes.data, bwh.ctypes.data, bwc.ctypes.data) != 0:
        return None
    return n.value, fwh, fwc[: m.value], bwh, bwc[: m.value]


def ref_tarjan(g: Graph):
    R = ref_lib()
    out = np.zeros(max(g.n, 1), np.uint32)
    ns = R.kref_tarjan(g.n, g.m, g.fwh, g.fwc, out)
    return out[: g.n].copy(), ns * 1e-9
