"""ORACLE - test infrastructure only.

ctypes wrapper of liboracle.so (oracle.cpp): the independent backtracking
matcher and the CPU restatement of the reference GpSM pipeline. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this package;
the product (gpsm_b200, libgpsm.so) never does.
"""
import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

REF_OK, REF_EMPTY_INIT, REF_EMPTY_REFINE, REF_EMPTY_JOIN = 0, 1, 2, 3
REF_DISCONNECTED, REF_NO_EDGES, REF_EMPTY_CEDGE = 4, 5, 6

vp, u32, u64, i32, i64 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_int64
_SIG = {
    "oracle_enumerate": (i64, [u32, vp, vp, vp, u32, vp, u32, vp, u64, vp, u64]),
    "oracle_enumerate_ordered": (i64, [u32, vp, vp, vp, u32, vp, u32, vp, vp, u64, vp, u64, u64, vp, vp, vp]),
    "oracle_label_index": (vp, [u32, vp, vp, vp, C.c_int]),
    "oracle_label_index_free": (None, [vp]),
    "oracle_ref_plan": (vp, [u32, vp, vp, vp, u32, vp, u32, vp, vp]),
    "oracle_ref_free": (None, [vp]),
    "oracle_ref_info": (None, [vp, vp, vp, vp, vp]),
    "oracle_ref_edges": (None, [vp, vp, vp]),
    "oracle_ref_order": (None, [vp, vp]),
    "oracle_ref_cand": (C.c_int, [vp, C.c_int, vp]),
    "oracle_ref_cedge_sizes": (None, [vp, vp, vp, vp, vp]),
    "oracle_ref_cedge_len": (u64, [vp, u32, C.c_int]),
    "oracle_ref_cedge_copy": (None, [vp, u32, C.c_int, vp]),
    "oracle_ref_steps": (None, [vp, vp, vp, vp]),
    "oracle_ref_mapping": (None, [vp, vp, vp]),
    "oracle_ref_join": (i64, [vp, C.c_int, u64, vp, vp, u64, vp, u64]),
    "oracle_ref_verify": (C.c_int, [vp, vp, vp, u64, vp]),
    "oracle_cpu_pipeline": (C.c_double, [u32, vp, vp, vp, u32, vp, vp, vp, vp, C.c_int, u64, vp, C.c_double]),
}
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        for k, (r, a) in _SIG.items():
            f = getattr(lib, k)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(vp)


class Graph:
    """Undirected data graph for the oracle: CSR with sorted lists."""

    def __init__(self, n, offsets, cols, labels, edges=None):
        self.n = int(n)
        self.offsets = offsets
        self.cols = cols
        self.labels = labels
        self.edges = edges


class Query:
    """Query graph: labels [qn] and (from, to) edges [qm, 2] in file order."""

    def __init__(self, labels, edges):
        self.labels = np.ascontiguousarray(labels, dtype=np.uint32)
        self.edges = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 2)

    @property
    def n(self):
        return int(self.labels.shape[0])

    @property
    def m(self):
        return int(self.edges.shape[0])


def csr_from_edges(n, edges):
    """The undirected CSR of graph/Graph.cpp:30-65 built with numpy, written
    apart from the engine's own CSR code: both directions of every edge,
    each list sorted ascending, parallel edges kept."""
    e = np.asarray(edges, dtype=np.uint64).reshape(-1, 2)
    src = np.concatenate([e[:, 0], e[:, 1]])
    dst = np.concatenate([e[:, 1], e[:, 0]])
    key = np.sort((src << np.uint64(32)) | dst)
    cols = (key & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    deg = np.bincount((key >> np.uint64(32)).astype(np.int64), minlength=n)
    offsets = np.zeros(n + 1, np.uint32)
    np.cumsum(deg, out=offsets[1:])
    return offsets, cols


def graph_from_edges(n, edges, labels):
    off, cols = csr_from_edges(n, edges)
    return Graph(n, off, cols, np.ascontiguousarray(labels, dtype=np.uint32),
                 np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 2))


_GEN_SIG = {
    "gpsm_gen_er": (C.c_int, [u32, u64, u64, vp]),
    "gpsm_gen_rmat": (C.c_int, [C.c_int, u64, C.c_double, C.c_double, C.c_double, u64, vp]),
    "gpsm_gen_labels": (C.c_int, [u32, u32, C.c_double, u64, vp]),
    "gpsm_gen_query": (i64, [u32, vp, vp, vp, u32, C.c_int, C.c_double, C.c_double, u64, vp, vp, vp]),
}


class _GenSource:
    """Workload source for gpsm_b200.workloads that never loads libgpsm.so:
    the seeded generators compiled into liboracle.so and the oracle's own
    CSR construction (csr_from_edges)."""

    name = "oracle"

    def lib(self):
        lib = load()
        if not getattr(lib, "_gen_declared", False):
            for k, (r, a) in _GEN_SIG.items():
                f = getattr(lib, k)
                f.restype = r
                f.argtypes = a
            lib._gen_declared = True
        return lib

    def csr(self, n, edges):
        return csr_from_edges(n, edges)


GEN_SOURCE = _GenSource()


def _u32(x):
    return np.ascontiguousarray(x, dtype=np.uint32)


def enumerate_embeddings(g, q, cap=1 << 62, rows=True, out_cap=None):
    """Sorted embeddings (rows indexed by query vertex) and their count."""
    lib = load()
    qe = _u32(q.edges).reshape(-1)
    if rows:
        if out_cap is None:
            cnt = lib.oracle_enumerate(g.n, _p(g.offsets), _p(g.cols), _p(g.labels), q.n, _p(_u32(q.labels)),
                                       q.m, _p(qe), cap, None, 0)
            out_cap = cnt
        out = np.zeros((max(out_cap, 1), q.n), dtype=np.uint32)
        cnt = lib.oracle_enumerate(g.n, _p(g.offsets), _p(g.cols), _p(g.labels), q.n, _p(_u32(q.labels)),
                                   q.m, _p(qe), cap, _p(out), out_cap)
        return out[: min(cnt, out_cap)], cnt
    cnt = lib.oracle_enumerate(g.n, _p(g.offsets), _p(g.cols), _p(g.labels), q.n, _p(_u32(q.labels)),
                               q.m, _p(qe), cap, None, 0)
    return None, cnt


class _LabelIndex:
    """Handle of the oracle's label-run index of one graph (freed with it)."""

    def __init__(self, g):
        self.lib = load()
        self.g = g  # keeps the CSR arrays alive
        self.h = self.lib.oracle_label_index(g.n, _p(g.offsets), _p(g.cols), _p(g.labels), os.cpu_count() or 1)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_label_index_free(self.h)
            self.h = None


_INDEX_LOCK = threading.Lock()


def label_index(g):
    """The oracle's label-run index of g, built once (by one thread) and
    kept on g."""
    with _INDEX_LOCK:
        li = getattr(g, "_oracle_label_index", None)
        if li is None:
            li = _LabelIndex(g)
            g._oracle_label_index = li
        return li


class WorkBoundHit(Exception):
    """The oracle's search visited its work bound before finishing."""


def enumerate_ordered(g, q, pos2id, cap=1 << 62, work_cap=0, rows=True, with_digest=False):
    """The first `cap` embeddings in the lexicographic order of their values
    taken in the vertex order pos2id (the order a join in that vertex order
    emits them), by backtracking from the definition. Returns (rows, count)
    or, with_digest, (rows, count, digest): rows (count, qn) with column p =
    query vertex pos2id[p] (None when rows=False); digest = rows_digest of
    all `count` rows, computed while searching. Raises WorkBoundHit when
    work_cap search steps (nodes and candidates examined) came first."""
    lib = load()
    qe = _u32(q.edges).reshape(-1)
    order = np.ascontiguousarray(pos2id, dtype=np.int32)
    out_cap = min(cap, 1 << 26) if rows else 0
    out = np.zeros((max(out_cap, 1), q.n), np.uint32) if rows else None
    partial = u64(0)
    dig = u64(0)
    li = label_index(g)  # held for the whole call
    cnt = lib.oracle_enumerate_ordered(g.n, _p(g.offsets), _p(g.cols), _p(g.labels), q.n, _p(_u32(q.labels)),
                                       q.m, _p(qe), _p(order), cap, _p(out), out_cap, work_cap, C.byref(partial),
                                       C.byref(dig), li.h)
    if cnt == -2:
        raise ValueError("pos2id is not a permutation of the query vertices")
    if cnt == -1:
        raise WorkBoundHit(f"work bound {work_cap} hit after {partial.value} rows")
    if rows and cnt > out_cap:
        raise ValueError("more rows than the output holds")
    r = out[:cnt] if rows else None
    return (r, cnt, dig.value) if with_digest else (r, cnt)


_M1, _M2 = np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)


def _fold(z):
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def rows_digest(rows, chunk=1 << 22):
    """Order-sensitive digest of a table (rows in order, columns in position
    order): sum over rows i of (i + 1) * hash(row i) mod 2^64, the hash a
    splitmix64-style fold of (value | position << 32). Same value as the
    digest enumerate_ordered computes while searching."""
    rows = np.asarray(rows)
    total = np.uint64(0)
    with np.errstate(over="ignore"):
        for a in range(0, rows.shape[0], chunk):
            blk = rows[a:a + chunk]
            h = np.full(blk.shape[0], 0x243F6A8885A308D3, np.uint64)
            for p in range(blk.shape[1]):
                h = _fold(h ^ (blk[:, p].astype(np.uint64) | (np.uint64(p) << np.uint64(32))))
            w = np.arange(a + 1, a + 1 + blk.shape[0], dtype=np.uint64)
            total = total + np.sum(h * w, dtype=np.uint64)
    return int(total)


class RefPlan:
    """CPU restatement of the reference pipeline for one (graph, query)."""

    def __init__(self, g, q):
        self.lib = load()
        self.g, self.q = g, q
        st = C.c_int32(0)
        self._ql = _u32(q.labels)
        self._qe = _u32(q.edges).reshape(-1)
        self.h = self.lib.oracle_ref_plan(g.n, _p(g.offsets), _p(g.cols), _p(g.labels), q.n, _p(self._ql),
                                          q.m, _p(self._qe), C.byref(st))
        self.status = st.value
        m, ns, de, no = u32(0), u32(0), i32(0), u32(0)
        self.lib.oracle_ref_info(self.h, C.byref(m), C.byref(ns), C.byref(de), C.byref(no))
        self.m, self.nsteps, self.defect, self.norder = m.value, ns.value, de.value, no.value

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_ref_free(self.h)
            self.h = None

    def edges(self):
        f = np.zeros(self.m, np.uint32)
        t = np.zeros(self.m, np.uint32)
        self.lib.oracle_ref_edges(self.h, _p(f), _p(t))
        return f, t

    def filter_order(self):
        o = np.zeros(self.norder, np.uint32)
        self.lib.oracle_ref_order(self.h, _p(o))
        return o

    def candidates(self, which=1):
        out = np.zeros((self.q.n, self.g.n), np.uint8)
        if self.lib.oracle_ref_cand(self.h, which, _p(out)) != 0:
            return None
        return out.astype(bool)

    def cedge_sizes(self):
        sf = np.zeros(self.m, np.uint64)
        nf = np.zeros(self.m, np.uint32)
        sr = np.zeros(self.m, np.uint64)
        nr = np.zeros(self.m, np.uint32)
        self.lib.oracle_ref_cedge_sizes(self.h, _p(sf), _p(nf), _p(sr), _p(nr))
        return sf, nf, sr, nr

    def cedge(self, e, rev=False):
        n = self.lib.oracle_ref_cedge_len(self.h, e, int(rev))
        out = np.zeros(n, np.uint32)
        self.lib.oracle_ref_cedge_copy(self.h, e, int(rev), _p(out))
        return out

    def steps(self):
        e = np.zeros(self.nsteps, np.uint32)
        mo = np.zeros(self.nsteps, np.int32)
        de = np.zeros(self.nsteps, np.int32)
        self.lib.oracle_ref_steps(self.h, _p(e), _p(mo), _p(de))
        return e, mo, de

    def mapping(self):
        a = np.zeros(self.q.n, np.int32)
        b = np.zeros(self.q.n, np.int32)
        self.lib.oracle_ref_mapping(self.h, _p(a), _p(b))
        return a, b  # id2pos, pos2id

    def join(self, injective=True, cap=1 << 62, rows=True, out_cap=None, work_cap=0):
        """(rows in table-column order or None, count, per-step row counts, capped)."""
        lv = np.zeros(max(self.nsteps, 1), np.uint64)
        capped = C.c_int(0)
        if rows:
            if out_cap is None:
                cnt = self.lib.oracle_ref_join(self.h, int(injective), cap, _p(lv), None, 0, C.byref(capped), work_cap)
                out_cap = cnt
            out = np.zeros((max(out_cap, 1), self.q.n), np.uint32)
            cnt = self.lib.oracle_ref_join(self.h, int(injective), cap, _p(lv), _p(out), out_cap,
                                           C.byref(capped), work_cap)
            return out[: min(cnt, out_cap)], cnt, lv[: self.nsteps], bool(capped.value)
        cnt = self.lib.oracle_ref_join(self.h, int(injective), cap, _p(lv), None, 0, C.byref(capped), work_cap)
        return None, cnt, lv[: self.nsteps], bool(capped.value)


DEADLINE_STOPPED = np.iinfo(np.int64).min


def cpu_pipeline(g, queries, threads=None, cap=1 << 62, deadline_s=0.0):
    """CPU port of the whole path over a query list: (counts, seconds).
    counts[k] == DEADLINE_STOPPED when the deadline stopped query k."""
    lib = load()
    threads = threads or os.cpu_count() or 1
    voff = np.zeros(len(queries) + 1, np.uint32)
    eoff = np.zeros(len(queries) + 1, np.uint64)
    for i, q in enumerate(queries):
        voff[i + 1] = voff[i] + q.n
        eoff[i + 1] = eoff[i] + q.m
    ql = np.concatenate([_u32(q.labels) for q in queries]) if queries else np.zeros(1, np.uint32)
    qe = np.concatenate([_u32(q.edges).reshape(-1) for q in queries]) if queries else np.zeros(2, np.uint32)
    qe = _u32(qe)
    counts = np.zeros(len(queries), np.int64)
    secs = lib.oracle_cpu_pipeline(g.n, _p(g.offsets), _p(g.cols), _p(g.labels), len(queries), _p(voff),
                                   _p(_u32(ql)), _p(eoff), _p(qe), threads, cap, _p(counts), float(deadline_s))
    return counts, secs
