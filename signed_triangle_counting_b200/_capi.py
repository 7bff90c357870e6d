"""ctypes declarations of include/stc.h and include/stc_synth.h.

The shared library is the in-tree ``libstc.so`` built by
``signed_triangle_counting_b200.build``.  Loading fails loudly when it is
missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libstc.so"

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
i8p = C.POINTER(C.c_int8)
i32p = C.POINTER(C.c_int32)
f32p = C.POINTER(C.c_float)


class stc_counts(C.Structure):
    _fields_ = [("t0", C.c_uint64), ("t1", C.c_uint64), ("t2", C.c_uint64), ("t3", C.c_uint64)]


class stc_edge_list(C.Structure):
    _fields_ = [("n", C.c_uint32), ("lines", C.c_uint64), ("m", C.c_uint64),
                ("src", u32p), ("dst", u32p), ("sign", i8p)]


class stc_forward_csr(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("offsets", u64p), ("edges", u32p),
                ("signs", i8p), ("fdeg", u32p), ("rank", u32p)]


class stc_graph(C.Structure):
    _fields_ = [("src", u32p), ("dst", u32p), ("sign", i8p), ("m", C.c_uint64)]


class stc_opts(C.Structure):
    _fields_ = [("strategy", C.c_uint32), ("dispatch", C.c_uint32), ("flags", C.c_uint32),
                ("reserved", C.c_uint32), ("stream", C.c_void_p)]


class stc_stats(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m_input", C.c_uint64), ("m_unique", C.c_uint64),
                ("m_forward", C.c_uint64), ("alg_bytes", C.c_uint64), ("triangles", C.c_uint64),
                ("ms_h2d", C.c_double), ("ms_dedup", C.c_double), ("ms_orient", C.c_double),
                ("ms_csr", C.c_double), ("ms_count", C.c_double), ("ms_total", C.c_double),
                ("kernel_launches", C.c_uint32), ("groups_replayed", C.c_uint32),
                ("probe_bytes", C.c_uint64)]


class stc_text_info(C.Structure):
    _fields_ = [("lines", C.c_uint64), ("n", C.c_uint32), ("reserved", C.c_uint32)]


class stc_tuning(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("hash_factor", C.c_uint32 * 3),
                ("unroll", C.c_uint32 * 3)]


class stc_synth_graph(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m", C.c_uint64), ("src", u32p), ("dst", u32p), ("sign", i8p)]


class stc_batch_spec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n", C.c_uint64), ("kind", C.c_uint32),
                ("rmat_scale", C.c_uint32), ("m_target", C.c_uint64), ("p_pos", C.c_double)]


# Status codes (stc_status).
STC_OK = 0
STC_ERR_INVALID_ARGUMENT = 1
STC_ERR_IO = 2
STC_ERR_CUDA = 3
STC_ERR_OUT_OF_MEMORY = 4
STC_ERR_LIMIT = 5
STC_ERR_DEVICE_TIMEOUT = 6
STC_ERR_NO_DEVICE = 7
STC_ERR_INTERNAL = 8

STRATEGY = {"auto": 0, "merge": 1, "hash": 2, "search": 3, "split": 4, "head": 5}
DISPATCH_CELLS = 1024
DISPATCH_FEATURES = 6
DISPATCH_MODEL_PARAMS = 197
DISPATCH_OUTPUTS = 5  # merge, hash, search, split, head
DISPATCH = {"fixed": 0, "learned": 1}
F_DEVICE_INPUT = 0x1
F_TIMING = 0x2
F_PERSISTENT = 0x8
MTX_ZERO_NEGATIVE = 0x1

# (name, restype, argtypes) for every exported function of include/*.h.
SIGNATURES = [
    ("stc_ctx_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    ("stc_ctx_destroy", None, [C.c_void_p]),
    ("stc_ctx_last_error", C.c_char_p, [C.c_void_p]),
    ("stc_ctx_last_stats", C.c_int, [C.c_void_p, C.POINTER(stc_stats)]),
    ("stc_ctx_trim", C.c_int, [C.c_void_p]),
    ("stc_status_string", C.c_char_p, [C.c_int]),
    ("stc_abi_version", C.c_int, []),
    ("stc_load_edge_list", C.c_int, [C.c_char_p, C.POINTER(stc_edge_list)]),
    ("stc_parse_edge_text", C.c_int, [C.c_char_p, C.c_uint64, C.POINTER(stc_edge_list)]),
    ("stc_free_edge_list", None, [C.POINTER(stc_edge_list)]),
    ("stc_load_mtx", C.c_int, [C.c_char_p, C.c_uint32, C.POINTER(stc_edge_list)]),
    ("stc_parse_mtx", C.c_int, [C.c_char_p, C.c_uint64, C.c_uint32, C.POINTER(stc_edge_list)]),
    ("stc_count", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                            C.POINTER(stc_opts), C.POINTER(stc_counts)]),
    ("stc_count_shard", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                  C.POINTER(stc_opts), C.c_uint32, C.c_uint32,
                                  C.POINTER(stc_counts), u64p]),
    ("stc_count_text", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(stc_opts),
                                 C.POINTER(stc_counts), C.POINTER(stc_text_info)]),
    ("stc_parse_edge_text_gpu", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(stc_opts),
                                          C.POINTER(stc_edge_list)]),
    ("stc_build_forward_csr", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_uint64, C.POINTER(stc_opts),
                                        C.POINTER(stc_forward_csr)]),
    ("stc_free_forward_csr", None, [C.POINTER(stc_forward_csr)]),
    ("stc_count_forward_csr", C.c_int, [C.c_void_p, C.POINTER(stc_forward_csr),
                                        C.POINTER(stc_opts), C.POINTER(stc_counts)]),
    ("stc_vertex_counts", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                    C.POINTER(stc_opts), u64p, C.c_uint64, u32p]),
    ("stc_count_batch", C.c_int, [C.c_void_p, C.POINTER(stc_graph), C.c_uint32,
                                  C.POINTER(stc_opts), C.POINTER(stc_counts)]),
    ("stc_count_batch_packed", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         u64p, C.c_uint32, C.POINTER(stc_opts),
                                         C.POINTER(stc_counts)]),
    ("stc_count_oriented_csr_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                                 C.c_uint64, C.c_void_p, C.POINTER(stc_counts)]),
    ("stc_record_bucket_times", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_uint64, C.POINTER(stc_opts), u64p, u64p,
                                          C.POINTER(stc_counts)]),
    ("stc_dispatch_features", C.c_int, [f32p]),
    ("stc_dispatcher_train", C.c_int, [C.c_void_p, f32p, f32p, f32p, C.c_uint32, C.c_uint32,
                                       C.c_float, C.c_float, C.c_uint64, f32p, f32p]),
    ("stc_ctx_set_dispatch_model", C.c_int, [C.c_void_p, f32p, u8p]),
    ("stc_dispatch_tables", C.c_int, [C.c_void_p, C.c_uint32, u8p]),
    ("stc_ctx_set_tuning", C.c_int, [C.c_void_p, C.POINTER(stc_tuning)]),
    ("stc_ctx_get_tuning", C.c_int, [C.c_void_p, C.POINTER(stc_tuning)]),
    ("stc_autotune", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                               C.POINTER(stc_opts), C.c_uint32, C.POINTER(stc_tuning)]),
    ("stc_synth_rmat_device", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint64,
                                        C.c_uint64, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    # include/stc_synth.h
    ("stc_synth_er", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_double,
                               C.POINTER(stc_synth_graph)]),
    ("stc_synth_rmat", C.c_int, [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.POINTER(stc_synth_graph)]),
    ("stc_synth_delaunay", C.c_int, [C.c_uint64, C.c_uint64, C.c_double, C.c_double,
                                     C.POINTER(stc_synth_graph)]),
    ("stc_synth_skew", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint64,
                                 C.c_uint64, C.c_double, C.POINTER(stc_synth_graph)]),
    ("stc_synth_batch_specs", C.c_int, [C.c_uint64, C.c_uint32, C.POINTER(stc_batch_spec)]),
    ("stc_synth_batch_graph", C.c_int, [C.POINTER(stc_batch_spec), C.POINTER(stc_synth_graph)]),
    ("stc_synth_batch_packed", C.c_int, [C.POINTER(stc_batch_spec), C.c_uint32, C.c_uint32,
                                         C.POINTER(stc_synth_graph), u64p]),
    ("stc_synth_workload", C.c_int, [C.c_int, C.c_uint32, C.POINTER(stc_synth_graph)]),
    ("stc_synth_workload_seed", C.c_uint64, [C.c_int]),
    ("stc_synth_set_threads", None, [C.c_uint32]),
    ("stc_synth_free", None, [C.POINTER(stc_synth_graph)]),
]

_lib = None


def lib() -> C.CDLL:
    """Loads libstc.so once; raises if the native library is absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m signed_triangle_counting_b200.build`"
                " (the counting path has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
