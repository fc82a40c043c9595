"""ctypes binding of libgpsm.so (declared in include/gpsm.h).

The library is the product: every matching call goes through its C ABI and
runs on the GPU. If the shared object is missing, loading raises instead of
falling back to anything else.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpsm.so")

GPSM_OK = 0
ERRORS = {
    -1: "GPSM_ERR_INVALID",
    -2: "GPSM_ERR_CUDA",
    -3: "GPSM_ERR_NOMEM",
    -4: "GPSM_ERR_NOT_FOUND",
    -5: "GPSM_ERR_BUDGET",
    -6: "GPSM_ERR_TIMEOUT",
    -7: "GPSM_ERR_NODEV",
    -8: "GPSM_ERR_STATE",
}


class GpsmError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({code})")


_lib = None

vp = C.c_void_p
u32, u64, i32, i64, f64 = C.c_uint32, C.c_uint64, C.c_int32, C.c_int64, C.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "gpsm_gen_er": (C.c_int, [u32, u64, u64, vp]),
    "gpsm_gen_rmat": (C.c_int, [C.c_int, u64, f64, f64, f64, u64, vp]),
    "gpsm_gen_labels": (C.c_int, [u32, u32, f64, u64, vp]),
    "gpsm_csr_from_edges": (C.c_int, [u32, u64, vp, vp, vp]),
    "gpsm_gen_query": (i64, [u32, vp, vp, vp, u32, C.c_int, f64, f64, u64, vp, vp, vp]),
    "gpsm_last_error": (C.c_char_p, []),
    "gpsm_text_open": (C.c_int, [C.c_char_p, vp]),
    "gpsm_text_count": (C.c_int, [vp, vp]),
    "gpsm_text_graph_info": (C.c_int, [vp, u32, vp, vp, vp]),
    "gpsm_text_graph_read": (C.c_int, [vp, u32, vp, vp, vp]),
    "gpsm_text_close": (C.c_int, [vp]),
    "gpsm_text_write": (C.c_int, [C.c_char_p, C.c_int, i32, u32, vp, u64, vp, vp, C.c_int]),
    "gpsm_init": (C.c_int, [C.c_int]),
    "gpsm_init_ex": (C.c_int, [C.c_int, u64]),
    "gpsm_shutdown": (C.c_int, []),
    "gpsm_engine_create": (C.c_int, [C.c_int, u64, vp]),
    "gpsm_engine_destroy": (C.c_int, [vp]),
    "gpsm_graph_upload": (C.c_int, [vp, vp, vp, u32, vp]),
    "gpsm_graph_free": (C.c_int, [vp]),
    "gpsm_graph_info": (C.c_int, [vp, vp, vp, vp]),
    "gpsm_graph_edge_table": (C.c_int, [vp, vp, vp]),
    "gpsm_graph_set_directed": (C.c_int, [vp, u64, vp, vp]),
    "gpsm_graph_build": (C.c_int, [vp, u64, vp, u32, vp]),
    "gpsm_graph_download": (C.c_int, [vp, vp, vp]),
    "gpsm_match_ex": (C.c_int, [vp, u32, vp, u32, vp, vp, vp, vp, vp, vp]),
    "gpsm_engine_match": (C.c_int, [vp, vp, u32, vp, u32, vp, vp, vp, vp, vp, vp]),
    "gpsm_match": (C.c_int, [vp, u32, vp, u32, vp, u64, vp, vp, vp, vp]),
    "gpsm_free": (None, [vp]),
    "gpsm_host_pool_stats": (None, [vp, vp, vp, vp]),
    "gpsm_debug_filter": (C.c_int, [vp, u32, vp, u32, vp, vp, vp, vp, vp, vp, vp]),
    "gpsm_match_batch": (C.c_int, [vp, vp, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "gpsm_flush_l2": (C.c_int, [vp, u64]),
    "gpsm_debug_skew_scan_tickets": (C.c_int, [vp, u32]),
    "gpsm_select_vertices": (C.c_int, [vp, vp, vp, u32, u32, u32, vp, vp]),
    "gpsm_select_vertices_static": (C.c_int, [vp, vp, u32, u32, u32, vp, vp, vp]),
    "gpsm_last_levels": (C.c_int, [vp, u32, vp, vp, vp]),
    "gpsm_match_batch_parallel": (C.c_int, [vp, u32, vp, vp, vp, vp, vp, vp, u32, u64, vp, vp, vp, vp]),
    "gpsm_server_create": (C.c_int, [vp, u32, u64, u64, vp, i32, vp]),
    "gpsm_server_submit": (C.c_int, [vp, u32, vp, u32, vp, vp]),
    "gpsm_server_wait": (C.c_int, [vp, u64, f64, vp, vp, vp]),
    "gpsm_server_wait_any": (C.c_int, [vp, f64, vp, vp, vp, vp]),
    "gpsm_server_stats": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "gpsm_server_destroy": (C.c_int, [vp]),
    "gpsm_set_tuning": (C.c_int, [vp]),
    "gpsm_get_tuning": (C.c_int, [vp]),
    "gpsm_model_params": (C.c_int, []),
    "gpsm_model_create": (C.c_int, [C.c_int, u64, vp]),
    "gpsm_model_destroy": (C.c_int, [vp]),
    "gpsm_model_set": (C.c_int, [vp, vp]),
    "gpsm_model_get": (C.c_int, [vp, vp]),
    "gpsm_model_train": (C.c_int, [vp, vp, vp, u32, u32, u32, C.c_float, u64, vp]),
    "gpsm_model_grad": (C.c_int, [vp, vp, vp, u32, vp, vp]),
    "gpsm_model_predict": (C.c_int, [vp, vp, u32, vp]),
    "gpsm_order_features": (C.c_int, [vp, u32, vp, u32, vp, vp, vp, vp, vp, vp]),
}

GPSM_ORDER_PLAIN, GPSM_ORDER_GIVEN, GPSM_ORDER_LEARNED = 0, 1, 2
GPSM_F_COUNT_ONLY, GPSM_F_KEEP_ON_DEVICE, GPSM_F_DIRECTED, GPSM_F_LARGEST_FIRST = 1, 2, 4, 8


class MatchOpts(C.Structure):
    _fields_ = [("cap", u64), ("order_mode", i32), ("pad", i32), ("order", vp),
                ("level_bytes", u64), ("result_rows", u64), ("flags", u32), ("pad2", u32),
                ("model", vp), ("memory_budget", u64), ("work_cap", u64), ("edge_labels", vp)]


class MatchInfo(C.Structure):
    _fields_ = [("rows", u64), ("cols", u32), ("capped", i32), ("empty_filter", i32), ("pad", i32),
                ("device_ms", f64), ("filter_ms", f64), ("join_ms", f64),
                ("expand_launches", u64), ("filter_launches", u64), ("alg_bytes_join", u64),
                ("expand_ms", f64), ("plan_ms", f64), ("predicted_work", f64), ("predicted_peak", f64),
                ("order_fallback", i32), ("aborted", i32), ("predicted_work_plain", f64),
                ("order_attempts", u32), ("pad2", u32), ("cands_scanned", u64), ("cut_steps", u64)]


class Tuning(C.Structure):
    _fields_ = [("heavy_degree", u32), ("ext_blocks_per_sm", u32), ("step_cands", u64), ("level_bytes", u64),
                ("slots", u32), ("scan_spin_limit", u32), ("race_share", u64),
                ("ext_items", u32), ("filter_team", u32), ("explore_team", u32), ("pad", u32)]


class RequestInfo(C.Structure):
    _fields_ = [("status", i32), ("capped", i32), ("rows", u64), ("submit_ms", f64), ("start_ms", f64),
                ("admit_ms", f64), ("end_ms", f64), ("device_ms", f64), ("admitted_bytes", u64)]


class BatchInfo(C.Structure):
    _fields_ = [("device_ms", f64), ("expand_ms", f64), ("filter_ms", f64), ("rows", u64), ("launches", u64),
                ("expand_launches", u64), ("alg_bytes_join", u64), ("join_steps", u64)]


def load(path=None):
    """Load libgpsm.so once and declare every exported signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"libgpsm.so not built at {p}; run gpsm_b200.build.build()")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    """Raw data pointer of a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(vp)


def check(code, what):
    if code < 0:
        msg = what
        if _lib is not None:
            err = _lib.gpsm_last_error()
            if err:
                msg = f"{what} ({err.decode(errors='replace')})"
        raise GpsmError(int(code), msg)
    return code


def u32a(x):
    return np.ascontiguousarray(x, dtype=np.uint32)


class _Block:
    """Frees one malloc'd result block of the library when collected."""

    def __init__(self, lib, addr):
        self.lib, self.addr = lib, addr

    def __del__(self):
        if self.addr:
            self.lib.gpsm_free(C.c_void_p(self.addr))
            self.addr = 0


def take_rows(lib, addr, nrows, ncols):
    """A (nrows, ncols) uint32 array over a result block the library handed
    over (no copy); the block is freed with the last view of it."""
    if not addr:
        return np.zeros((0, ncols), np.uint32)
    if nrows * ncols == 0:
        lib.gpsm_free(C.c_void_p(addr))
        return np.zeros((0, ncols), np.uint32)
    buf = (C.c_uint32 * (nrows * ncols)).from_address(addr)
    buf._owner = _Block(lib, addr)
    return np.frombuffer(buf, dtype=np.uint32).reshape(nrows, ncols)
