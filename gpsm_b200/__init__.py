"""gpsm_b200: B200-native subgraph matching behind the GpSM host API.

Every call below goes through libgpsm.so's C ABI (include/gpsm.h) and runs
hand-written sm_100a kernels. There is no CPU fallback: without a GPU the
matching entry points raise GpsmError(GPSM_ERR_NODEV).

    from gpsm_b200 import init, DeviceGraph, match
    init(0)
    dg = DeviceGraph(graph)                 # offsets / cols / labels, uploaded once
    out = match(dg, query, cap=10**7)       # plain (reference) join order
    out.rows                                # (R, qn) uint32, table-column order
    out.embeddings()                        # (R, qn) indexed by query vertex
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import GpsmError  # noqa: F401

__all__ = ["init", "shutdown", "DeviceGraph", "Engine", "match", "match_batch", "flush_l2", "MatchOutput",
           "debug_filter", "GpsmError", "pack_queries"]


def init(device=0, arena_bytes=0):
    """Select the device and create the default engine (Match::initGPU)."""
    lib = _lib.load()
    _lib.check(lib.gpsm_init_ex(device, arena_bytes), "gpsm_init")


def shutdown():
    lib = _lib.load()
    _lib.check(lib.gpsm_shutdown(), "gpsm_shutdown")


class DeviceGraph:
    """A data graph uploaded once to device memory (graph handle)."""

    def __init__(self, graph):
        lib = _lib.load()
        self._lib = lib
        self.graph = graph
        self.n = int(graph.n)
        h = _lib.vp()
        off = _lib.u32a(graph.offsets)
        cols = _lib.u32a(graph.cols) if len(graph.cols) else np.zeros(1, np.uint32)
        lab = _lib.u32a(graph.labels)
        _lib.check(lib.gpsm_graph_upload(_lib.ptr(off), _lib.ptr(cols), _lib.ptr(lab), self.n, C.byref(h)),
                   "gpsm_graph_upload")
        self.handle = h

    def free(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self._lib.gpsm_graph_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Engine:
    """An additional engine (own stream and workspace) on one device."""

    def __init__(self, device=0, arena_bytes=0):
        lib = _lib.load()
        self._lib = lib
        h = _lib.vp()
        _lib.check(lib.gpsm_engine_create(device, arena_bytes, C.byref(h)), "gpsm_engine_create")
        self.handle = h

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self._lib.gpsm_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class MatchOutput:
    rows: np.ndarray  # (R, qn) uint32 in table-column order (None when count only)
    count: int
    id_map: np.ndarray  # id2pos: query vertex -> column
    pos2id: np.ndarray  # column -> query vertex
    capped: bool
    empty_filter: bool
    info: dict

    def embeddings(self):
        """Rows re-indexed by query vertex (column j = query vertex j)."""
        if self.rows is None:
            return None
        if self.rows.shape[0] == 0:
            return self.rows
        return np.ascontiguousarray(self.rows[:, self.id_map])


def _query_arrays(query):
    ql = _lib.u32a(query.labels)
    qe = _lib.u32a(np.asarray(query.edges).reshape(-1)) if query.m else np.zeros(2, np.uint32)
    return ql, qe


def match(dgraph, query, cap=None, order=None, count_only=False, keep_on_device=False, engine=None,
          level_bytes=0, result_rows=0):
    """Match one query (Match::match). order: None = the reference's plain
    join order, else pos2id (a connected vertex order)."""
    lib = _lib.load()
    qn = query.n
    ql, qe = _query_arrays(query)
    opts = _lib.MatchOpts()
    opts.cap = int(cap or 0)
    order_arr = None
    if order is not None:
        order_arr = np.ascontiguousarray(order, dtype=np.int32)
        opts.order_mode = _lib.GPSM_ORDER_GIVEN
        opts.order = order_arr.ctypes.data
    opts.level_bytes = int(level_bytes)
    opts.result_rows = int(result_rows)
    opts.flags = (_lib.GPSM_F_COUNT_ONLY if count_only else 0) | (_lib.GPSM_F_KEEP_ON_DEVICE if keep_on_device else 0)
    info = _lib.MatchInfo()
    id_map = np.zeros(qn, np.int32)
    pos2id = np.zeros(qn, np.int32)
    out = _lib.vp()
    out_arg = None if count_only else C.byref(out)
    eng = engine.handle if engine is not None else None
    rc = lib.gpsm_engine_match(eng, dgraph.handle, qn, _lib.ptr(ql), query.m, _lib.ptr(qe), C.byref(opts),
                               out_arg, _lib.ptr(id_map), _lib.ptr(pos2id), C.byref(info))
    _lib.check(rc, "gpsm_match")
    rows = None
    if not count_only:
        nrows = int(info.rows)
        if out.value:
            buf = (C.c_uint32 * (nrows * qn)).from_address(out.value) if nrows * qn else None
            rows = np.frombuffer(buf, dtype=np.uint32).copy().reshape(nrows, qn) if buf is not None else \
                np.zeros((0, qn), np.uint32)
            lib.gpsm_free(out)
        else:
            rows = np.zeros((0, qn), np.uint32)
    d = {k: getattr(info, k) for k, _ in _lib.MatchInfo._fields_ if k not in ("pad",)}
    return MatchOutput(rows, int(info.rows), id_map, pos2id, bool(info.capped), bool(info.empty_filter), d)


def debug_filter(dgraph, query, with_candidates=False):
    """Filter-stage products for comparison with the reference restatement."""
    lib = _lib.load()
    qn, m, N = query.n, query.m, dgraph.n
    ql, qe = _query_arrays(query)
    cc = np.zeros(qn, np.uint32)
    sf = np.zeros(max(m, 1), np.uint64)
    sr = np.zeros(max(m, 1), np.uint64)
    fo = np.zeros(qn, np.uint32)
    po = np.zeros(qn, np.int32)
    bits = np.zeros((qn, N), np.uint8) if with_candidates else None
    rc = lib.gpsm_debug_filter(dgraph.handle, qn, _lib.ptr(ql), m, _lib.ptr(qe), _lib.ptr(cc), _lib.ptr(sf),
                               _lib.ptr(sr), _lib.ptr(fo), _lib.ptr(po), _lib.ptr(bits))
    _lib.check(rc, "gpsm_debug_filter")
    return dict(empty=(rc == 1), cand_count=cc, size_fwd=sf[:m], size_rev=sr[:m], filter_order=fo,
                plain_pos2id=po, candidates=None if bits is None else bits.astype(bool))


def pack_queries(queries):
    """Concatenated query arrays for the batch entry point."""
    nq = len(queries)
    voff = np.zeros(nq + 1, np.uint32)
    eoff = np.zeros(nq + 1, np.uint64)
    for i, q in enumerate(queries):
        voff[i + 1] = voff[i] + q.n
        eoff[i + 1] = eoff[i] + q.m
    ql = _lib.u32a(np.concatenate([np.asarray(q.labels, np.uint32) for q in queries]))
    qe = [np.asarray(q.edges, np.uint32).reshape(-1) for q in queries if q.m]
    qe = _lib.u32a(np.concatenate(qe)) if qe else np.zeros(2, np.uint32)
    return voff, ql, eoff, qe


def match_batch(dgraph, queries, cap=None, orders=None, engine=None, packed=None, level_bytes=0):
    """Match queries back to back on one engine (rows stay on the device).
    Returns (counts, capped, per-query device ms, batch info dict)."""
    lib = _lib.load()
    voff, ql, eoff, qe = packed if packed is not None else pack_queries(queries)
    nq = len(voff) - 1
    opts = _lib.MatchOpts()
    opts.cap = int(cap or 0)
    opts.level_bytes = int(level_bytes)
    ords = None
    if orders is not None:
        ords = np.ascontiguousarray(np.concatenate([np.asarray(o, np.int32) for o in orders]), np.int32)
        opts.order_mode = _lib.GPSM_ORDER_GIVEN
    counts = np.zeros(nq, np.uint64)
    capped = np.zeros(nq, np.int32)
    qms = np.zeros(nq, np.float64)
    info = _lib.BatchInfo()
    eng = engine.handle if engine is not None else None
    rc = lib.gpsm_match_batch(eng, dgraph.handle, nq, _lib.ptr(voff), _lib.ptr(ql), _lib.ptr(eoff), _lib.ptr(qe),
                              C.byref(opts), _lib.ptr(ords), _lib.ptr(counts), _lib.ptr(capped), _lib.ptr(qms),
                              C.byref(info))
    _lib.check(rc, "gpsm_match_batch")
    d = {k: getattr(info, k) for k, _ in _lib.BatchInfo._fields_}
    return counts, capped.astype(bool), qms, d


def flush_l2(nbytes=256 << 20, engine=None):
    lib = _lib.load()
    eng = engine.handle if engine is not None else None
    _lib.check(lib.gpsm_flush_l2(eng, int(nbytes)), "gpsm_flush_l2")
