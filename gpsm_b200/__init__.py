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
           "debug_filter", "GpsmError", "pack_queries", "Model", "order_features", "last_levels", "Server", "host_pool_stats",
           "set_tuning", "get_tuning"]


import json as _json
import os as _os

TUNING_FILE = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "data", "tuning.json")


def init(device=0, arena_bytes=0, tuning_file=TUNING_FILE):
    """Select the device and create the default engine (Match::initGPU).
    Applies the autotuner's choices when tuning_file exists."""
    lib = _lib.load()
    if tuning_file and _os.path.exists(tuning_file):
        set_tuning(**_json.load(open(tuning_file)).get("choice", {}))
    _lib.check(lib.gpsm_init_ex(device, arena_bytes), "gpsm_init")


def set_tuning(**kw):
    """Process-wide launch choices: heavy_degree, ext_blocks_per_sm,
    step_cands, level_bytes, slots, race_share, scan_spin_limit, ext_items,
    filter_team, explore_team (unset or 0 = unchanged)."""
    lib = _lib.load()
    t = _lib.Tuning()
    for k, v in kw.items():
        if k in dict(_lib.Tuning._fields_):
            setattr(t, k, int(v))
    _lib.check(lib.gpsm_set_tuning(C.byref(t)), "gpsm_set_tuning")


def get_tuning():
    lib = _lib.load()
    t = _lib.Tuning()
    _lib.check(lib.gpsm_get_tuning(C.byref(t)), "gpsm_get_tuning")
    return {k: getattr(t, k) for k, _ in _lib.Tuning._fields_ if k != "pad"}


def shutdown():
    lib = _lib.load()
    _lib.check(lib.gpsm_shutdown(), "gpsm_shutdown")


class DeviceGraph:
    """A data graph uploaded once to device memory (graph handle).
    build_on_device=True builds the CSR on the GPU from graph.edges."""

    def __init__(self, graph, build_on_device=False):
        lib = _lib.load()
        self._lib = lib
        self.graph = graph
        self.n = int(graph.n)
        h = _lib.vp()
        lab = _lib.u32a(graph.labels)
        if build_on_device:
            e = _lib.u32a(np.asarray(graph.edges).reshape(-1))
            _lib.check(lib.gpsm_graph_build(_lib.ptr(e), len(e) // 2, _lib.ptr(lab), self.n, C.byref(h)),
                       "gpsm_graph_build")
        else:
            off = _lib.u32a(graph.offsets)
            cols = _lib.u32a(graph.cols) if len(graph.cols) else np.zeros(1, np.uint32)
            _lib.check(lib.gpsm_graph_upload(_lib.ptr(off), _lib.ptr(cols), _lib.ptr(lab), self.n, C.byref(h)),
                       "gpsm_graph_upload")
        self.handle = h

    def download(self):
        """(offsets, cols) of the device CSR."""
        nnz = C.c_uint64()
        self._lib.gpsm_graph_info(self.handle, None, C.byref(nnz), None)
        off = np.zeros(self.n + 1, np.uint32)
        cols = np.zeros(max(nnz.value, 1), np.uint32)
        _lib.check(self._lib.gpsm_graph_download(self.handle, _lib.ptr(off), _lib.ptr(cols)), "gpsm_graph_download")
        return off, cols[: nnz.value]

    def edge_table(self):
        """(slots, longest probe) of the edge table built at upload; slots
        0 when it was not built (the joins then search the lists)."""
        slots, probe = C.c_uint64(), C.c_uint32()
        _lib.check(self._lib.gpsm_graph_edge_table(self.handle, C.byref(slots), C.byref(probe)),
                   "gpsm_graph_edge_table")
        return slots.value, probe.value

    def set_directed(self, edges, labels=None):
        """Directed, labelled data edges (pairs (from, to) as in the file)
        for directed matching (IO::verify's test on the device)."""
        e = _lib.u32a(np.asarray(edges).reshape(-1))
        lab = None if labels is None else _lib.u32a(labels)
        _lib.check(self._lib.gpsm_graph_set_directed(self.handle, len(e) // 2, _lib.ptr(e), _lib.ptr(lab)),
                   "gpsm_graph_set_directed")

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
          level_bytes=0, result_rows=0, model=None, memory_budget=0, work_cap=0, directed=False,
          edge_labels=None):
    """Match one query (Match::match). order: None = the reference's plain
    join order, a pos2id list (a connected vertex order), or "learned" (the
    order chosen by `model`, falling back to the plain order when its
    predicted peak table exceeds memory_budget bytes)."""
    lib = _lib.load()
    qn = query.n
    ql, qe = _query_arrays(query)
    opts = _lib.MatchOpts()
    opts.cap = int(cap or 0)
    order_arr = None
    if isinstance(order, str) and order == "learned":
        if model is None:
            raise ValueError("order='learned' needs a model")
        opts.order_mode = _lib.GPSM_ORDER_LEARNED
        opts.model = model.handle
    elif order is not None:
        order_arr = np.ascontiguousarray(order, dtype=np.int32)
        opts.order_mode = _lib.GPSM_ORDER_GIVEN
        opts.order = order_arr.ctypes.data
    opts.memory_budget = int(memory_budget)
    opts.work_cap = int(work_cap)
    elab = None
    if directed and edge_labels is not None:
        elab = _lib.u32a(edge_labels)
        opts.edge_labels = elab.ctypes.data
    opts.level_bytes = int(level_bytes)
    opts.result_rows = int(result_rows)
    opts.flags = ((_lib.GPSM_F_COUNT_ONLY if count_only else 0) | (_lib.GPSM_F_KEEP_ON_DEVICE if keep_on_device else 0)
                  | (_lib.GPSM_F_DIRECTED if directed else 0))
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
        rows = _lib.take_rows(lib, out.value, int(info.rows), qn)
    d = {k: getattr(info, k) for k, _ in _lib.MatchInfo._fields_ if k not in ("pad", "pad2")}
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


def match_batch(dgraph, queries, cap=None, orders=None, engine=None, packed=None, level_bytes=0, slots=1,
                model=None, slot_arena=0, work_cap=0):
    """Match queries back to back (rows stay on the device); slots > 1 runs
    them on that many engine slots at once (continuous batching); orders:
    None (plain), "learned" (model) or a list of pos2id per query; work_cap:
    candidates a query's joins may scan (0 = no bound).
    Returns (counts, capped, per-query device ms, batch info dict): capped
    is True where the embedding cap or the work cap stopped a query; the
    info dict's "aborted" counts the work-cap stops and "stop" holds the
    per-query codes (0 complete, 1 embedding cap, 2 work cap)."""
    lib = _lib.load()
    voff, ql, eoff, qe = packed if packed is not None else pack_queries(queries)
    nq = len(voff) - 1
    opts = _lib.MatchOpts()
    opts.cap = int(cap or 0)
    opts.work_cap = int(work_cap)
    opts.level_bytes = int(level_bytes)
    ords = None
    if isinstance(orders, str) and orders == "learned":
        opts.order_mode = _lib.GPSM_ORDER_LEARNED
        opts.model = model.handle
    elif orders is not None:
        ords = np.ascontiguousarray(np.concatenate([np.asarray(o, np.int32) for o in orders]), np.int32)
        opts.order_mode = _lib.GPSM_ORDER_GIVEN
    counts = np.zeros(nq, np.uint64)
    capped = np.zeros(nq, np.int32)
    qms = np.zeros(nq, np.float64)
    info = _lib.BatchInfo()
    eng = engine.handle if engine is not None else None
    if slots > 1:
        rc = lib.gpsm_match_batch_parallel(dgraph.handle, nq, _lib.ptr(voff), _lib.ptr(ql), _lib.ptr(eoff),
                                           _lib.ptr(qe), C.byref(opts), _lib.ptr(ords), slots, int(slot_arena),
                                           _lib.ptr(counts), _lib.ptr(capped), _lib.ptr(qms), C.byref(info))
    else:
        rc = lib.gpsm_match_batch(eng, dgraph.handle, nq, _lib.ptr(voff), _lib.ptr(ql), _lib.ptr(eoff), _lib.ptr(qe),
                                  C.byref(opts), _lib.ptr(ords), _lib.ptr(counts), _lib.ptr(capped), _lib.ptr(qms),
                                  C.byref(info))
    _lib.check(rc, "gpsm_match_batch")
    d = {k: getattr(info, k) for k, _ in _lib.BatchInfo._fields_}
    d["aborted"] = int((capped == 2).sum())
    d["stop"] = capped.copy()
    return counts, capped.astype(bool), qms, d


def flush_l2(nbytes=256 << 20, engine=None):
    lib = _lib.load()
    eng = engine.handle if engine is not None else None
    _lib.check(lib.gpsm_flush_l2(eng, int(nbytes)), "gpsm_flush_l2")


class Model:
    """The learned join-order MLP (16 -> 64 -> 64 -> 1, BF16 weights, FP32
    accumulation) on one device; training and inference run on the GPU."""

    def __init__(self, device=0, seed=0, params=None):
        lib = _lib.load()
        self._lib = lib
        self.n_params = lib.gpsm_model_params()
        h = _lib.vp()
        _lib.check(lib.gpsm_model_create(device, seed, C.byref(h)), "gpsm_model_create")
        self.handle = h
        if params is not None:
            self.set(params)

    def set(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == self.n_params
        _lib.check(self._lib.gpsm_model_set(self.handle, _lib.ptr(p)), "gpsm_model_set")

    def get(self):
        p = np.zeros(self.n_params, np.float32)
        _lib.check(self._lib.gpsm_model_get(self.handle, _lib.ptr(p)), "gpsm_model_get")
        return p

    def train(self, x, y, epochs=30, batch=2048, lr=2e-3, seed=0):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = C.c_float(0)
        _lib.check(self._lib.gpsm_model_train(self.handle, _lib.ptr(x), _lib.ptr(y), len(y), epochs, batch, lr, seed,
                                              C.byref(loss)), "gpsm_model_train")
        return loss.value

    def grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_float(0)
        _lib.check(self._lib.gpsm_model_grad(self.handle, _lib.ptr(x), _lib.ptr(y), len(y), _lib.ptr(g),
                                             C.byref(loss)), "gpsm_model_grad")
        return loss.value, g

    def predict(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros(len(x), np.float32)
        _lib.check(self._lib.gpsm_model_predict(self.handle, _lib.ptr(x), len(x), _lib.ptr(y)), "gpsm_model_predict")
        return y

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self._lib.gpsm_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def order_features(dgraph, query, filt, pos2id):
    """Features of every join step of the order pos2id ((n-1, 16) float32),
    from debug_filter()'s statistics."""
    lib = _lib.load()
    ql, qe = _query_arrays(query)
    out = np.zeros((max(query.n - 1, 1), 16), np.float32)
    cc = np.ascontiguousarray(filt["cand_count"], np.uint32)
    sf = np.ascontiguousarray(filt["size_fwd"], np.uint64)
    sr = np.ascontiguousarray(filt["size_rev"], np.uint64)
    if sf.size == 0:
        sf = np.zeros(1, np.uint64)
        sr = np.zeros(1, np.uint64)
    po = np.ascontiguousarray(pos2id, np.int32)
    _lib.check(lib.gpsm_order_features(dgraph.handle, query.n, _lib.ptr(ql), query.m, _lib.ptr(qe), _lib.ptr(cc),
                                       _lib.ptr(sf), _lib.ptr(sr), _lib.ptr(po), _lib.ptr(out)), "gpsm_order_features")
    return out[: query.n - 1]


def last_levels(n, engine=None):
    """(rows extended, candidates scanned, rows produced) per table width 0..n
    of the engine's last match."""
    lib = _lib.load()
    a = np.zeros(n + 1, np.uint64)
    b = np.zeros(n + 1, np.uint64)
    c = np.zeros(n + 1, np.uint64)
    eng = engine.handle if engine is not None else None
    _lib.check(lib.gpsm_last_levels(eng, n, _lib.ptr(a), _lib.ptr(b), _lib.ptr(c)), "gpsm_last_levels")
    return a, b, c


def host_pool_stats():
    """The page-locked result-block pool: blocks held, bytes pinned, blocks
    added since the process started and the host ms spent pinning them."""
    lib = _lib.load()
    v = [C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_double()]
    lib.gpsm_host_pool_stats(*[C.byref(x) for x in v])
    return dict(blocks=v[0].value, pinned_bytes=v[1].value, grown=v[2].value, grow_ms=v[3].value)


class Server:
    """Request loop over `slots` engine slots: submit() returns at once,
    wait() blocks until the request is done. Requests are admitted to their
    joins when their predicted join memory fits memory_budget bytes."""

    def __init__(self, dgraph, slots=4, memory_budget=0, slot_arena=0, cap=None, order=None, model=None,
                 collect_rows=False, work_cap=0, result_rows=0, largest_first=False):
        lib = _lib.load()
        self._lib = lib
        opts = _lib.MatchOpts()
        opts.cap = int(cap or 0)
        opts.work_cap = int(work_cap)
        opts.result_rows = int(result_rows)  # device rows per copy to the host (0: 4 Mi)
        if largest_first:  # a free slot takes the queued request with the most edges
            opts.flags |= _lib.GPSM_F_LARGEST_FIRST
        if order == "learned":
            opts.order_mode = _lib.GPSM_ORDER_LEARNED
            opts.model = model.handle
        self._model = model  # keep alive
        h = _lib.vp()
        _lib.check(lib.gpsm_server_create(dgraph.handle, slots, int(memory_budget), int(slot_arena), C.byref(opts),
                                          1 if collect_rows else 0, C.byref(h)), "gpsm_server_create")
        self.handle = h
        self.collect = collect_rows
        self._qn = {}  # ticket -> query vertices, for requests not yet collected

    def submit(self, query):
        ql, qe = _query_arrays(query)
        t = C.c_uint64(0)
        _lib.check(self._lib.gpsm_server_submit(self.handle, query.n, _lib.ptr(ql), query.m, _lib.ptr(qe),
                                                C.byref(t)), "gpsm_server_submit")
        self._qn[t.value] = query.n
        return t.value, query.n

    def wait(self, ticket, timeout=-1.0, raise_on_error=True):
        """The request's info (status, times, rows, ...); with
        raise_on_error=False a failed request returns its info (status < 0,
        "error" = the engine's text) instead of raising."""
        tid, qn = ticket
        info = _lib.RequestInfo()
        info.status = 1  # stays 1 when the call fails before filling info (bad ticket, timeout)
        out = _lib.vp()
        idm = np.zeros(qn, np.int32)
        rc = self._lib.gpsm_server_wait(self.handle, tid, float(timeout), C.byref(info),
                                        C.byref(out) if self.collect else None, _lib.ptr(idm))
        return self._result(rc, info, out, idm, tid, qn, raise_on_error, "gpsm_server_wait")

    def wait_any(self, timeout=-1.0, raise_on_error=True):
        """(ticket, info) of the first finished request not yet collected,
        in completion order (same info as wait())."""
        info = _lib.RequestInfo()
        info.status = 1
        out = _lib.vp()
        idm = np.zeros(128, np.int32)
        t = C.c_uint64(0)
        rc = self._lib.gpsm_server_wait_any(self.handle, float(timeout), C.byref(t), C.byref(info),
                                            C.byref(out) if self.collect else None, _lib.ptr(idm))
        if rc != 0 and info.status == 1:
            _lib.check(rc, "gpsm_server_wait_any")
        qn = self._qn.get(t.value, 0)
        return (t.value, qn), self._result(rc, info, out, idm[:qn].copy(), t.value, qn, raise_on_error,
                                           "gpsm_server_wait_any")

    def _result(self, rc, info, out, idm, tid, qn, raise_on_error, what):
        if info.status != 1:  # collected (a timeout leaves the request outstanding)
            self._qn.pop(tid, None)
        if rc != 0 and (raise_on_error or info.status == 1):
            _lib.check(rc, what)
        if rc != 0:
            return {k: getattr(info, k) for k, _ in _lib.RequestInfo._fields_} | {
                "error": self._lib.gpsm_last_error().decode(errors="replace")}
        d = {k: getattr(info, k) for k, _ in _lib.RequestInfo._fields_}
        if self.collect:
            # the table in join-column order (as the reference returns it);
            # column id_map[u] holds query vertex u: table[:, id_map] is the
            # embeddings in query-vertex order
            d["table"] = _lib.take_rows(self._lib, out.value, int(info.rows), qn)
            d["id_map"] = idm
        return d

    def stats(self):
        v = [C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32(), C.c_uint32()]
        _lib.check(self._lib.gpsm_server_stats(self.handle, *[C.byref(x) for x in v]), "gpsm_server_stats")
        return dict(in_use=v[0].value, peak_in_use=v[1].value, budget=v[2].value, queued=v[3].value,
                    active=v[4].value)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self._lib.gpsm_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
