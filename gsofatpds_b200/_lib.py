"""ctypes binding of libgsofa.so (the C-ABI declared in include/gsofa.h).

The library is built in-tree (``make -C gsofatpds_b200/csrc``); importing
this module without it raises immediately -- there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(HERE, "libgsofa.so")
CLI_PATH = os.path.join(HERE, "gsofa_cli")

OK = 0
ERR_ARG = 1
ERR_IO = 2
ERR_OOM_BUDGET = 3
ERR_TIMEOUT = 4
ERR_OVERFLOW = 5
ERR_CUDA = 6
ERR_UNSUPPORTED = 7
ERR_BUSY = 8
ERR_SCRATCH = 9

SUPERNODES = 1 << 0
L_ROW_STATS = 1 << 1
PATTERN = 1 << 2
DIGESTS = 1 << 3
FORCE_GLOBAL_BITMAP = 1 << 30
NO_MERGE = 1 << 29
DEBUG_QUEUE_CAP = 1 << 28
NO_CHAIN = 1 << 27

# Every function the header declares (checked by the CPU test-suite).
EXPORTS = [
    "gsofa_opts_default", "gsofa_create", "gsofa_destroy", "gsofa_last_error",
    "gsofa_status_string", "gsofa_set_stream", "gsofa_memory_used", "gsofa_load_csr",
    "gsofa_load_csr_files", "gsofa_matrix_info", "gsofa_matrix_destroy",
    "gsofa_factor_symbolic", "gsofa_factor_batch", "gsofa_result_counts",
    "gsofa_result_row_counts", "gsofa_result_digests", "gsofa_result_supernodes",
    "gsofa_result_lmask", "gsofa_result_pattern_u", "gsofa_result_pattern_l",
    "gsofa_result_destroy", "gsofa_symbfact_min_id", "gsofa_factor_symbolic_noalloc",
    "gsofa_autotune", "gsofa_batch_create", "gsofa_batch_run", "gsofa_batch_result",
    "gsofa_batch_destroy", "gsofa_server_create", "gsofa_server_submit", "gsofa_server_poll",
    "gsofa_server_wait", "gsofa_server_ticket_info", "gsofa_server_get_stats",
    "gsofa_server_destroy", "gsofa_server_last_error", "gsofa_autotune_batch",
    "gsofa_write_csr_binary", "gsofa_read_csr_binary", "gsofa_convert_dat_to_binary",
    "gsofa_load_csr_binary", "gsofa_result_supernodal", "gsofa_order_nd", "gsofa_order_hybrid", "gsofa_matrix_permute",
    "gsofa_order_wait_selftest",
]


class Opts(ctypes.Structure):
    _fields_ = [("max_supernode_size", ctypes.c_int32),
                ("threads_per_source", ctypes.c_int32),
                ("sources_in_flight", ctypes.c_int32),
                ("flags", ctypes.c_uint32),
                ("bu_alpha", ctypes.c_int32),
                ("bu_beta", ctypes.c_int32),
                ("heavy_row", ctypes.c_int32),
                ("bu_min_source", ctypes.c_int32),
                ("chunk_sources", ctypes.c_int32),
                ("cached_closures", ctypes.c_int32),
                ("chain_wait_us", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class Counts(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("fill_count", ctypes.c_uint64), ("nnz_l", ctypes.c_uint64),
                ("nnz_u", ctypes.c_uint64), ("nnz_lu", ctypes.c_uint64),
                ("n_supernodes", ctypes.c_int64), ("edges_alg", ctypes.c_uint64),
                ("vertices_alg", ctypes.c_uint64), ("edges_traversed", ctypes.c_uint64),
                ("ms_device", ctypes.c_double), ("ms_traverse", ctypes.c_double),
                ("sources_chained", ctypes.c_uint64)]


class OrderStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int32), ("splits", ctypes.c_int32),
                ("separator_vertices", ctypes.c_int64), ("max_separator", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("ms", ctypes.c_double)]


class TicketInfo(ctypes.Structure):
    _fields_ = [("t_submit_ms", ctypes.c_double), ("t_admit_ms", ctypes.c_double),
                ("t_publish_ms", ctypes.c_double), ("t_done_ms", ctypes.c_double),
                ("footprint_bytes", ctypes.c_uint64), ("status", ctypes.c_int32),
                ("n", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64),
                ("items_published", ctypes.c_uint64), ("bytes_in_use", ctypes.c_uint64),
                ("peak_bytes", ctypes.c_uint64), ("fixed_bytes", ctypes.c_uint64),
                ("grid", ctypes.c_int32), ("block", ctypes.c_int32),
                ("max_in_flight", ctypes.c_int32), ("reserved", ctypes.c_int32)]


_lib = None


def load():
    """Load libgsofa.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SO_PATH):
        raise OSError("libgsofa.so is not built (run: make -C %s/csrc)" % HERE)
    L = ctypes.CDLL(SO_PATH)
    vp = ctypes.c_void_p
    i32, i64, u32 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32
    sig = {
        "gsofa_opts_default": [ctypes.POINTER(Opts)],
        "gsofa_create": [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(vp)],
        "gsofa_destroy": [vp],
        "gsofa_set_stream": [vp, vp],
        "gsofa_memory_used": [vp, ctypes.POINTER(ctypes.c_size_t)],
        "gsofa_load_csr": [vp, i32, i64, vp, vp, vp, ctypes.POINTER(vp)],
        "gsofa_load_csr_files": [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                 ctypes.POINTER(vp)],
        "gsofa_matrix_info": [vp, ctypes.POINTER(i32), ctypes.POINTER(i64)],
        "gsofa_matrix_destroy": [vp],
        "gsofa_factor_symbolic": [vp, vp, ctypes.POINTER(Opts), ctypes.POINTER(vp)],
        "gsofa_factor_batch": [vp, ctypes.POINTER(vp), i32, ctypes.POINTER(Opts), ctypes.POINTER(vp)],
        "gsofa_result_counts": [vp, ctypes.POINTER(Counts)],
        "gsofa_result_row_counts": [vp, vp, vp, vp, vp],
        "gsofa_result_digests": [vp, vp, vp, vp],
        "gsofa_result_supernodes": [vp, vp, vp, i64, ctypes.POINTER(i64)],
        "gsofa_result_lmask": [vp, vp],
        "gsofa_result_pattern_u": [vp, vp, vp, i64],
        "gsofa_result_pattern_l": [vp, vp, vp, i64],
        "gsofa_result_destroy": [vp],
        "gsofa_autotune": [vp, vp, ctypes.POINTER(Opts)],
        "gsofa_autotune_batch": [vp, ctypes.POINTER(vp), i32, ctypes.POINTER(Opts)],
        "gsofa_write_csr_binary": [ctypes.c_char_p, i32, i64, vp, vp, vp],
        "gsofa_read_csr_binary": [ctypes.c_char_p, ctypes.POINTER(i32), ctypes.POINTER(i64), vp, vp,
                                  vp],
        "gsofa_convert_dat_to_binary": [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                        ctypes.c_char_p],
        "gsofa_load_csr_binary": [vp, ctypes.c_char_p, ctypes.POINTER(vp)],
        "gsofa_result_supernodal": [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64),
                                    vp, vp, vp, vp, vp],
        "gsofa_order_nd": [vp, vp, i32, i32, vp, ctypes.POINTER(OrderStats)],
        "gsofa_order_hybrid": [vp, vp, i32, vp, ctypes.POINTER(OrderStats)],
        "gsofa_matrix_permute": [vp, vp, vp, ctypes.POINTER(vp)],
        "gsofa_order_wait_selftest": [vp, ctypes.c_double],
        "gsofa_batch_create": [vp, ctypes.POINTER(vp), i32, ctypes.POINTER(Opts), ctypes.POINTER(vp)],
        "gsofa_batch_run": [vp],
        "gsofa_batch_result": [vp, i32, ctypes.POINTER(vp)],
        "gsofa_batch_destroy": [vp],
        "gsofa_factor_symbolic_noalloc": [vp, ctypes.POINTER(Opts), vp, vp, vp, vp, vp, vp, vp],
        "gsofa_server_create": [vp, ctypes.POINTER(Opts), i32, ctypes.c_size_t, ctypes.POINTER(vp)],
        "gsofa_server_submit": [vp, i32, i64, vp, vp, vp, ctypes.POINTER(ctypes.c_uint64)],
        "gsofa_server_poll": [vp, ctypes.c_uint64, ctypes.POINTER(vp)],
        "gsofa_server_wait": [vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(vp)],
        "gsofa_server_ticket_info": [vp, ctypes.c_uint64, ctypes.POINTER(TicketInfo)],
        "gsofa_server_get_stats": [vp, ctypes.POINTER(ServerStats)],
        "gsofa_server_destroy": [vp],
        "gsofa_symbfact_min_id": [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(i32), ctypes.POINTER(ctypes.c_uint64)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L.gsofa_last_error.argtypes = [vp]
    L.gsofa_last_error.restype = ctypes.c_char_p
    L.gsofa_server_last_error.argtypes = [vp]
    L.gsofa_server_last_error.restype = ctypes.c_char_p
    L.gsofa_status_string.argtypes = [ctypes.c_int]
    L.gsofa_status_string.restype = ctypes.c_char_p
    _ = u32
    _lib = L
    return L
