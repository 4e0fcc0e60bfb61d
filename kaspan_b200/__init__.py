"""kaspan_b200 -- strongly connected components on one NVIDIA B200.

Python view of the C ABI in include/kspn.h (libkspn.so, built from
kaspan_b200/csrc by ``python -m kaspan_b200.build``).  There is no CPU
fallback: every call runs the CUDA library, and importing the bindings fails
loudly when the library is missing.

Whole path (the reference's ``kaspan::scc(bidi_graph_part_view, vertex_t*)``,
kaspan/scc/scc.hpp:21-25):

    ids = kaspan_b200.scc(n, fw_head, fw_csr, bw_head, bw_csr)  # numpy, host
    ctx.scc_device(n, m, fwh, fwc, bwh, bwc, out)                # torch cuda

Output: ids[v] = minimum vertex id of v's strongly connected component.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkspn.so")

NOALLOC_MAX_N = 1 << 20  # KSPN_NOALLOC_MAX_N
MLP_PARAMS = 1377
MLP_FEATURES = 8
PIPELINE_FAST = 0
PIPELINE_REFERENCE = 1
PIPELINE_HPC_LIKE = 2
PIPELINE_HPC_TRIM_EX = 3
PIPELINE_ISPAN_LIKE = 4
PIPELINE_TRIM_EX = 5
PIPELINE_TRIM_EX_LIGHT_RESIDUAL = 6
PIPELINE_TRIM_EX_RESIDUAL = 7
# the reference's entry points: kaspan::scc and its variants (variant/*.hpp)
PIPELINES = {"scc": PIPELINE_REFERENCE, "hpc_like": PIPELINE_HPC_LIKE, "hpc_trim_ex": PIPELINE_HPC_TRIM_EX,
             "ispan_like": PIPELINE_ISPAN_LIKE, "trim_ex": PIPELINE_TRIM_EX,
             "trim_ex_light_residual": PIPELINE_TRIM_EX_LIGHT_RESIDUAL, "trim_ex_residual": PIPELINE_TRIM_EX_RESIDUAL}
UNDECIDED = 0xFFFFFFFF

STATUS = {
    0: "KSPN_OK",
    1: "KSPN_ERR_INVALID_ARGUMENT",
    2: "KSPN_ERR_INVALID_GRAPH",
    3: "KSPN_ERR_OOM",
    4: "KSPN_ERR_TIMEOUT",
    5: "KSPN_ERR_CUDA",
    6: "KSPN_ERR_NO_DEVICE",
    7: "KSPN_ERR_INTERNAL",
}

PHASES = ["trim_first", "trim", "fwbw", "trim_normal", "label", "trim2", "residual", "canon"]
KERNEL_CLASSES = ["expand", "bottom_up", "trim", "stream"]


class Options(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("pipeline", C.c_int32),
        ("trim2", C.c_int32),
        ("validate", C.c_int32),
        ("bu_enter_div", C.c_uint32),
        ("bu_leave_div", C.c_uint32),
        ("max_levels", C.c_uint32),
        ("max_label_iters", C.c_uint32),
        ("max_rounds", C.c_uint32),
        ("profile", C.c_int32),
        ("trace", C.c_int32),
        ("learned_pivot", C.c_int32),
        ("wait_limit", C.c_uint32),
        ("drop_barrier", C.c_uint32),
        ("aw_exact_after", C.c_uint32),
        ("learned_seeds", C.c_int32),
    ]


class LevelTrace(C.Structure):
    _fields_ = [
        ("backward", C.c_uint32),
        ("bottom_up", C.c_uint32),
        ("frontier", C.c_uint32),
        ("discovered", C.c_uint32),
        ("frontier_edges", C.c_uint64),
        ("scanned", C.c_uint64),
        ("candidates", C.c_uint64),
        ("ms", C.c_float),
        ("pad", C.c_uint32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("m", C.c_uint64),
        ("decided", C.c_uint64 * 8),
        ("ms", C.c_double * 8),
        ("ms_total", C.c_double),
        ("edges_scanned", C.c_uint64),
        ("pivot", C.c_uint32),
        ("levels_fw", C.c_uint32),
        ("levels_bw", C.c_uint32),
        ("levels_bottom_up", C.c_uint32),
        ("label_calls", C.c_uint32),
        ("rounds", C.c_uint32),
        ("kernel_launches", C.c_uint64),
        ("kernel_ms", C.c_double * 4),
        ("kernel_bytes", C.c_uint64 * 4),
        ("kernel_calls", C.c_uint64 * 4),
        ("trace_levels", C.c_uint32),
        ("trace", LevelTrace * 32),
        ("search_marks", C.c_uint32),
        ("search_phase", C.c_uint32 * 128),
        ("search_ns", C.c_uint64 * 128),
        ("resident_ms", C.c_double),
        ("resident_bytes", C.c_uint64),
        ("resident_rows", C.c_uint64),
        ("resident_edges", C.c_uint64),
        ("resident_bitmap_passes", C.c_uint32),
        ("resident_pad", C.c_uint32),
        ("heavy_cut_rows", C.c_uint32),
        ("heavy_fixups", C.c_uint32),
        ("heavy_trim_seeds", C.c_uint32),
        ("trim_worklist", C.c_uint32),
        ("fwbw_joint", C.c_uint32),
        ("search_worklist", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {
            "n": self.n,
            "m": self.m,
            "decided": {p: int(self.decided[i]) for i, p in enumerate(PHASES)},
            "ms": {p: float(self.ms[i]) for i, p in enumerate(PHASES)},
            "ms_total": self.ms_total,
            "edges_scanned": int(self.edges_scanned),
            "pivot": self.pivot,
            "levels_fw": self.levels_fw,
            "levels_bw": self.levels_bw,
            "levels_bottom_up": self.levels_bottom_up,
            "label_calls": self.label_calls,
            "rounds": self.rounds,
            "kernel_launches": int(self.kernel_launches),
            "heavy": {"cut_rows": self.heavy_cut_rows, "fixups": self.heavy_fixups, "trim_seeds": self.heavy_trim_seeds},
            "trim_worklist": self.trim_worklist,
            "fwbw_joint": self.fwbw_joint,
            "search_worklist": self.search_worklist,
            "kernels": {k: {"ms": float(self.kernel_ms[i]), "bytes": int(self.kernel_bytes[i]), "calls": int(self.kernel_calls[i])}
                        for i, k in enumerate(KERNEL_CLASSES)},
            "trace": [{"dir": "bw" if t.backward else "fw", "mode": "bu" if t.bottom_up else "td", "frontier": t.frontier,
                       "discovered": t.discovered, "frontier_edges": int(t.frontier_edges), "scanned": int(t.scanned),
                       "candidates": int(t.candidates), "ms": round(float(t.ms), 4)}
                      for t in self.trace[: min(self.trace_levels, 32)]],
            "search_marks": [(int(self.search_phase[i]), int(self.search_ns[i])) for i in range(min(self.search_marks, 128))],
            "resident": {"ms": float(self.resident_ms), "bytes": int(self.resident_bytes), "rows": int(self.resident_rows),
                         "edges": int(self.resident_edges), "bitmap_passes": int(self.resident_bitmap_passes)},
        }


class KspnError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {detail}")


# every symbol include/kspn.h declares, with its ctypes signature
_P = C.c_void_p
_u32, _u64, _i32 = C.c_uint32, C.c_uint64, C.c_int
SIGNATURES = {
    "kspn_options_default": (_i32, [_P]),
    "kspn_options_size": (C.c_size_t, []),
    "kspn_stats_size": (C.c_size_t, []),
    "kspn_strerror": (C.c_char_p, [_i32]),
    "kspn_last_error": (C.c_char_p, [_P]),
    "kspn_context_create": (_i32, [_i32, _P]),
    "kspn_context_create_on_stream": (_i32, [_i32, _P, _P]),
    "kspn_context_destroy": (_i32, [_P]),
    "kspn_context_synchronize": (_i32, [_P]),
    "kspn_context_launches": (_u64, [_P]),
    "kspn_scc": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_scc_device": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_trim_1_first": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P]),
    "kspn_forward_backward_search": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _u32, _P]),
    "kspn_trim_1_normal": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_label_search": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _i32, _P, _P]),
    "kspn_trim_1_exhaustive_first": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_trim_1_fixpoint": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_set_pivot_model": (_i32, [_P, _P]),
    "kspn_mlp_features": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _u32, _P, _P]),
    "kspn_mlp_forward": (_i32, [_P, _u32, _P, _P, _P]),
    "kspn_mlp_gradient": (_i32, [_P, _u32, _P, _P, _P, _P, _P]),
    "kspn_mlp_adam": (_i32, [_P, _P, _P, _P, _P, C.c_float, _i32]),
    "kspn_residual": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P]),
    "kspn_trim_2": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_normalise": (_i32, [_P, _u32, _P]),
    "kspn_normalise_noalloc": (_i32, [_u32, _P, _P]),
    "kspn_transpose": (_i32, [_P, _u32, _u64, _P, _P, _P, _P]),
    "kspn_shard_trim_first": (_i32, [_P, _u32, _u32, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_shard_pivot": (_i32, [_P, _u32, _u32, _P, _P, _P, _P, _P]),
    "kspn_shard_search_begin": (_i32, [_P, _u32, _u32, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_shard_expand": (_i32, [_P, _u32, _u32, _P, _P, _P, _u32, _P, _P, _P, _P, _u32, _P, _P, _u32, _u32, _P, _P, _P, _P]),
    "kspn_shard_receive": (_i32, [_P, _u32, _u32, _P, _u32, _P, _P, _P, _u32, _P]),
    "kspn_shard_scc_min": (_i32, [_P, _u32, _u32, _P, _P, _P]),
    "kspn_shard_finalize": (_i32, [_P, _u32, _P, _P, _P, _P, _u32, _P]),
    "kspn_shard_residual": (_i32, [_P, _u32, _u32, _P, _P, _P, _P, _P, _P, _u64, _P]),
    "kspn_upload_transpose": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _u64]),
    "kspn_gen_gnm": (_i32, [_P, _u32, _u64, _u64, _P, _P]),
    "kspn_gen_rmat": (_i32, [_P, _i32, _u64, _u64, _u64, _u64, _u64, _i32, _P, _P]),
    "kspn_gen_rgg": (_i32, [_P, _u32, _u64, _u32, _u64, _P, _P, _u64, _P]),
    "kspn_build_csr": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P]),
    "kspn_batch_options_default": (None, [_P]),
    "kspn_scc_batched": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _P, _P]),
    "kspn_batch_shape": (None, [_u32, _u64, _u32, _u32, C.c_float, C.c_float, _P, _P]),
    "kspn_gen_batch": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P]),
    "kspn_batch_localize": (_i32, [_P, _u32, _u64, _P, _P, _P]),
    "kspn_manifest_read": (_i32, [C.c_char_p, _P]),
    "kspn_manifest_load": (_i32, [_P, _P, _P, _P, _P, _P]),
    "kspn_manifest_write": (_i32, [C.c_char_p, C.c_char_p, _u32, _u64, _P, _P, _P, _P, _u32, _u32, _i32, _i32, _i32]),
    "kspn_autotune": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _u32, _P, _P]),
    "kspn_autotune_batched": (_i32, [_P, _u32, _u64, _P, _P, _P, _P, _P, _P, _P, _u32, _P, _P]),
}


class Manifest(C.Structure):
    """kspn_manifest (include/kspn.h)."""
    _fields_ = [("schema_version", C.c_uint32), ("big_endian", C.c_int32), ("node_count", C.c_uint64), ("edge_count", C.c_uint64),
                ("self_loops", C.c_int32), ("duplicate_edges", C.c_int32), ("head_bytes", C.c_uint32), ("csr_bytes", C.c_uint32),
                ("graph_code", C.c_char * 64), ("graph_name", C.c_char * 128), ("fw_head_path", C.c_char * 1024),
                ("fw_csr_path", C.c_char * 1024), ("bw_head_path", C.c_char * 1024), ("bw_csr_path", C.c_char * 1024)]


def manifest_read(path: str) -> Manifest:
    """Parse a manifest file (host only)."""
    mf = Manifest()
    rc = lib().kspn_manifest_read(path.encode(), C.byref(mf))
    if rc:
        raise KspnError(rc, f"manifest_read: {path}")
    return mf


def manifest_write(directory: str, name: str, n: int, fw_head, fw_csr, bw_head, bw_csr, head_bytes: int = 8, csr_bytes: int = 4,
                   big_endian: bool = False, self_loops: bool = False, duplicate_edges: bool = False) -> str:
    """Write host arrays (numpy u64 heads, u32 ids) in the manifest format; returns the manifest path."""
    fw_head = np.ascontiguousarray(fw_head, np.uint64)
    bw_head = np.ascontiguousarray(bw_head, np.uint64)
    fw_csr = np.ascontiguousarray(fw_csr, np.uint32)
    bw_csr = np.ascontiguousarray(bw_csr, np.uint32)
    m = int(fw_head[n]) if n else 0
    rc = lib().kspn_manifest_write(directory.encode(), name.encode(), n, m, fw_head.ctypes.data, fw_csr.ctypes.data if fw_csr.size else None,
                                   bw_head.ctypes.data, bw_csr.ctypes.data if bw_csr.size else None, head_bytes, csr_bytes,
                                   int(big_endian), int(self_loops), int(duplicate_edges))
    if rc:
        raise KspnError(rc, f"manifest_write: {directory}/{name}")
    return os.path.join(directory, name + ".manifest")


class TuneReport(C.Structure):
    """kspn_tune_report (include/kspn.h)."""
    _fields_ = [("candidates", C.c_uint32), ("default_ms", C.c_float), ("best_ms", C.c_float), ("reserved", C.c_uint32 * 5)]


class BatchOptions(C.Structure):
    """kspn_batch_options (include/kspn.h)."""
    _fields_ = [("max_rounds", C.c_uint32), ("rem_tarjan", C.c_uint32), ("cluster_size", C.c_uint32), ("reserved0", C.c_uint32),
                ("cluster_min", C.c_uint64), ("search", C.c_uint32), ("route", C.c_uint32)]


class BatchStats(C.Structure):
    """kspn_batch_stats (include/kspn.h)."""
    _fields_ = [("graphs_small", C.c_uint32), ("graphs_large", C.c_uint32), ("fwbw_rounds", C.c_uint32),
                ("tarjan_smem", C.c_uint32), ("tarjan_serial", C.c_uint32), ("trim_levels", C.c_uint32),
                ("ms", C.c_float), ("graphs_cluster", C.c_uint32), ("cluster_size", C.c_uint32), ("phase_ms", C.c_float * 5),
                ("label_calls", C.c_uint32), ("reserved", C.c_uint32 * 1)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("reserved", "phase_ms")}
        d["phase_ms"] = dict(zip(("init", "trim", "pivot", "search", "remainder"), [round(x, 3) for x in self.phase_ms]))
        return d


def batch_shape(count: int, seed: int, log2_min: int = 8, log2_max: int = 18, deg_min: float = 0.8, deg_max: float = 6.0):
    """(n[count] uint32, draws[count] uint64) of the batch mix (host, deterministic)."""
    n = np.zeros(count, np.uint32)
    d = np.zeros(count, np.uint64)
    lib().kspn_batch_shape(count, seed, log2_min, log2_max, deg_min, deg_max, n.ctypes.data, d.ctypes.data)
    return n, d

_lib = None


def lib() -> C.CDLL:
    """The CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libkspn.so not found at {LIB_PATH}; build it with `python -m kaspan_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def default_pivot_model():
    """The shipped pivot model (numpy float32[MLP_PARAMS]) or None: trained
    by `python -m kaspan_b200.pivot_train` on the GPU."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pivot_model.npy")
    return np.load(path).astype(np.float32) if os.path.exists(path) else None


def default_options(**kw) -> Options:
    o = Options()
    lib().kspn_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _ptr(x) -> int | None:
    """Device/host address of a torch tensor or numpy array (None passes through)."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, int):
        return x
    raise TypeError(f"cannot take the address of {type(x)}")


class Context:
    """One kspn_context: a device, a stream, a reusable workspace."""

    def __init__(self, device: int = 0, stream=None):
        L = lib()
        h = C.c_void_p()
        if stream is None:
            rc = L.kspn_context_create(device, C.byref(h))
        else:
            s = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
            rc = L.kspn_context_create_on_stream(device, C.c_void_p(s), C.byref(h))
        if rc != 0:
            raise KspnError(rc, "context creation")
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            lib().kspn_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int, what: str):
        if rc != 0:
            detail = lib().kspn_last_error(self.h)
            raise KspnError(rc, f"{what}: {detail.decode() if detail else ''}")

    @property
    def launches(self) -> int:
        return int(lib().kspn_context_launches(self.h))

    def synchronize(self):
        self._check(lib().kspn_context_synchronize(self.h), "synchronize")

    # ---- whole path
    def scc(self, n, fw_head, fw_csr, bw_head=None, bw_csr=None, out=None, options=None, stats=None):
        """Host (numpy) arrays in, canonical ids out (numpy uint32[n])."""
        fw_head = np.ascontiguousarray(fw_head, dtype=np.uint64)
        m = int(fw_head[n]) if n else 0
        fw_csr = np.ascontiguousarray(fw_csr, dtype=np.uint32)
        if bw_head is not None:
            bw_head = np.ascontiguousarray(bw_head, dtype=np.uint64)
            bw_csr = np.ascontiguousarray(bw_csr, dtype=np.uint32)
        if out is None:
            out = np.empty(max(n, 1), np.uint32)
        opt = options if options is not None else default_options()
        rc = lib().kspn_scc(self.h, n, m, _ptr(fw_head), _ptr(fw_csr), _ptr(bw_head), _ptr(bw_csr), _ptr(out),
                            C.byref(opt), C.byref(stats) if stats is not None else None)
        self._check(rc, "kspn_scc")
        return out[:n]

    def scc_host_ptr(self, n, m, fwh, fwc, bwh, bwc, out, options=None, stats=None):
        """Host pointers (pinned torch tensors or numpy), result into `out`."""
        opt = options if options is not None else default_options()
        rc = lib().kspn_scc(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(out),
                            C.byref(opt), C.byref(stats) if stats is not None else None)
        self._check(rc, "kspn_scc")

    def scc_device(self, n, m, fwh, fwc, bwh, bwc, out, options=None, stats=None):
        """Device pointers (torch cuda tensors); result into `out`."""
        opt = options if options is not None else default_options()
        rc = lib().kspn_scc_device(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(out),
                                   C.byref(opt), C.byref(stats) if stats is not None else None)
        self._check(rc, "kspn_scc_device")

    # ---- phases (device pointers)
    def trim_1_first(self, n, m, fwh, bwh, und, scc_id) -> int:
        pivot = C.c_uint32()
        self._check(lib().kspn_trim_1_first(self.h, n, m, _ptr(fwh), _ptr(bwh), _ptr(und), _ptr(scc_id), C.byref(pivot)), "trim_1_first")
        return pivot.value

    def forward_backward_search(self, n, m, fwh, fwc, bwh, bwc, und, scc_id, pivot) -> int:
        d = C.c_uint32()
        self._check(lib().kspn_forward_backward_search(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(und), _ptr(scc_id), pivot, C.byref(d)), "forward_backward_search")
        return d.value

    def trim_1_normal(self, n, m, fwh, fwc, bwh, bwc, und, scc_id) -> int:
        d = C.c_uint32()
        self._check(lib().kspn_trim_1_normal(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(und), _ptr(scc_id), C.byref(d)), "trim_1_normal")
        return d.value

    def label_search(self, n, m, fwh, fwc, bwh, bwc, und, scc_id, rotation, label=None) -> int:
        d = C.c_uint32()
        self._check(lib().kspn_label_search(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(und), _ptr(scc_id), rotation, _ptr(label), C.byref(d)), "label_search")
        return d.value

    def trim_1_exhaustive_first(self, n, m, fwh, fwc, bwh, bwc, und, scc_id, outdeg, indeg) -> int:
        d = C.c_uint32()
        self._check(lib().kspn_trim_1_exhaustive_first(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(und), _ptr(scc_id), _ptr(outdeg), _ptr(indeg), C.byref(d)), "trim_1_exhaustive_first")
        return d.value

    def trim_1_fixpoint(self, n, m, fwh, fwc, bwh, bwc, und, scc_id) -> int:
        d = C.c_uint32()
        self._check(lib().kspn_trim_1_fixpoint(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(und), _ptr(scc_id), C.byref(d)), "trim_1_fixpoint")
        return d.value

    def trim_2(self, n, m, fwh, fwc, bwh, bwc, und, scc_id) -> int:
        d = C.c_uint32()
        self._check(lib().kspn_trim_2(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(und), _ptr(scc_id), C.byref(d)), "trim_2")
        return d.value

    def residual(self, n, m, fwh, fwc, und, scc_id):
        """(vertices decided, pieces left undecided)."""
        d, left = C.c_uint32(), C.c_uint32()
        self._check(lib().kspn_residual(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(und), _ptr(scc_id), C.byref(d), C.byref(left)), "residual")
        return d.value, left.value

    # ---- learned pivot (no reference counterpart)
    def set_pivot_model(self, params):
        """params: numpy float32[MLP_PARAMS], or None to remove the model."""
        if params is None:
            self._check(lib().kspn_set_pivot_model(self.h, None), "set_pivot_model")
            return
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == MLP_PARAMS
        self._check(lib().kspn_set_pivot_model(self.h, p.ctypes.data), "set_pivot_model")

    def mlp_features(self, n, m, fwh, fwc, bwh, bwc, vertices, features):
        self._check(lib().kspn_mlp_features(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), vertices.numel(), _ptr(vertices), _ptr(features)), "mlp_features")

    def mlp_forward(self, features, params, logits):
        self._check(lib().kspn_mlp_forward(self.h, features.shape[0], _ptr(features), _ptr(params), _ptr(logits)), "mlp_forward")

    def mlp_gradient(self, features, labels, params, grad, loss):
        self._check(lib().kspn_mlp_gradient(self.h, features.shape[0], _ptr(features), _ptr(labels), _ptr(params), _ptr(grad), _ptr(loss)), "mlp_gradient")

    def mlp_adam(self, params, grad, m, v, lr, step):
        self._check(lib().kspn_mlp_adam(self.h, _ptr(params), _ptr(grad), _ptr(m), _ptr(v), float(lr), int(step)), "mlp_adam")

    def normalise(self, n, scc_id):
        self._check(lib().kspn_normalise(self.h, n, _ptr(scc_id)), "normalise")

    def transpose(self, n, m, fwh, fwc, bwh, bwc):
        self._check(lib().kspn_transpose(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc)), "transpose")

    def upload_transpose(self, n, m, fwh_host, fwc_host, fwh, fwc, bwh, bwc, chunk_edges=0):
        """Host CSR (pinned torch tensors or numpy) -> device CSR + CSC, the
        CSC sorted chunk by chunk while the upload runs."""
        self._check(lib().kspn_upload_transpose(self.h, n, m, _ptr(fwh_host), _ptr(fwc_host), _ptr(fwh), _ptr(fwc),
                                                _ptr(bwh), _ptr(bwc), int(chunk_edges)), "upload_transpose")

    # ---- inputs
    def gen_gnm(self, n, draws, seed, src, dst):
        self._check(lib().kspn_gen_gnm(self.h, n, draws, seed, _ptr(src), _ptr(dst)), "gen_gnm")

    def gen_rmat(self, scale, draws, seed, ta, tab, tabc, permute, src, dst):
        self._check(lib().kspn_gen_rmat(self.h, scale, draws, seed, ta, tab, tabc, int(permute), _ptr(src), _ptr(dst)), "gen_rmat")

    def gen_rgg(self, n, seed, g, r2, src=None, dst=None, capacity=0) -> int:
        """Edge count of the RGG; writes the edges when src/dst are given."""
        m = C.c_uint64()
        self._check(lib().kspn_gen_rgg(self.h, n, seed, g, r2, _ptr(src) if src is not None else None,
                                       _ptr(dst) if dst is not None else None, capacity, C.byref(m)), "gen_rgg")
        return m.value

    # ---- batched path
    def scc_batched(self, count, n_total, vtx_off, fwh, fwc, bwh, bwc, out, options: "BatchOptions | None" = None) -> "BatchStats":
        st = BatchStats()
        self._check(lib().kspn_scc_batched(self.h, count, n_total, _ptr(vtx_off), _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(out),
                                           C.byref(options) if options is not None else None, C.byref(st)), "scc_batched")
        return st

    def manifest_load(self, mf: "Manifest", fwh, fwc, bwh, bwc):
        self._check(lib().kspn_manifest_load(self.h, C.byref(mf), _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc)), "manifest_load")

    def autotune(self, n, m, fwh, fwc, bwh, bwc, out, base: "Options | None" = None, reps: int = 3):
        """(best Options, TuneReport) for this graph (FAST pipeline settings)."""
        best, rep = Options(), TuneReport()
        self._check(lib().kspn_autotune(self.h, n, m, _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(out),
                                        C.byref(base) if base is not None else None, reps, C.byref(best), C.byref(rep)), "autotune")
        return best, rep

    def autotune_batched(self, count, n_total, vtx_off, fwh, fwc, bwh, bwc, out, base: "BatchOptions | None" = None, reps: int = 3):
        """(best BatchOptions, TuneReport) for this batch."""
        best, rep = BatchOptions(), TuneReport()
        self._check(lib().kspn_autotune_batched(self.h, count, n_total, _ptr(vtx_off), _ptr(fwh), _ptr(fwc), _ptr(bwh), _ptr(bwc), _ptr(out),
                                                C.byref(base) if base is not None else None, reps, C.byref(best), C.byref(rep)), "autotune_batched")
        return best, rep

    def gen_batch(self, count, seed, vtx_off, draw_off, src, dst, graph_ids=None):
        self._check(lib().kspn_gen_batch(self.h, count, seed, _ptr(vtx_off), _ptr(draw_off), _ptr(graph_ids), _ptr(src), _ptr(dst)), "gen_batch")

    def batch_localize(self, count, n_total, vtx_off, head, csr):
        self._check(lib().kspn_batch_localize(self.h, count, n_total, _ptr(vtx_off), _ptr(head), _ptr(csr)), "batch_localize")

    def build_csr(self, n, m_raw, src, dst, head, csr) -> int:
        m = C.c_uint64()
        self._check(lib().kspn_build_csr(self.h, n, m_raw, _ptr(src), _ptr(dst), _ptr(head), _ptr(csr), C.byref(m)), "build_csr")
        return m.value


def scc(n, fw_head, fw_csr, bw_head=None, bw_csr=None, options=None, device: int = 0):
    """One-shot host call: canonical SCC ids (numpy uint32[n])."""
    with Context(device) as ctx:
        return ctx.scc(n, fw_head, fw_csr, bw_head, bw_csr, options=options).copy()
