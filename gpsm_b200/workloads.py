"""Seeded synthetic data graphs and query sets for the five workload shapes.

No public dataset is named for this path and the reference's benchmark
datasets (script/run.sh: delaunay_n13, enron, gowalla, road_central) are not
available, so every workload is generated from a seed:

  small_er     ER G(10,000, 40,000), labels U{1..8}; 10 induced random-walk
               queries of 6 vertices
  rmat20       R-MAT(.57,.19,.19,.05) on 2^20 vertices, 16 Mi undirected edges,
               labels Zipf(1.0) over 1..32; 100 induced random-walk queries of
               12 vertices with average degree >= 2.5
  rmat20_mix   the rmat20 graph; 1,000 queries of 4..32 vertices, half tree
               (n-1 edges), half dense (extra induced edges kept with p=0.3)
  rmat22       R-MAT on 2^22 vertices, 64 Mi edges, Zipf(1.1) over 1..64;
               4,096 queries of 4..64 vertices (tree/dense mix)
  rmat24       R-MAT on 2^24 vertices, 256 Mi edges, Zipf(1.0) over 1..128;
               queries of 4..99 vertices, geometric with mean 16
Generation runs in compiled code (gen.cpp); this module only sequences it.
The default source is libgpsm.so (its generators and CSR builder). Test and
benchmark code that must not load the engine (the CPU reference arm) passes
oracle.GEN_SOURCE instead: the same generators compiled into liboracle.so,
with the oracle's own CSR construction; both sources give identical
workloads (tests/test_oracle.py checks it).
"""
from dataclasses import dataclass, field

import numpy as np

from . import _lib

MODE_INDUCED, MODE_TREE, MODE_DENSE = 0, 1, 2


@dataclass
class Graph:
    """Undirected data graph: CSR with sorted lists plus the edge list."""
    n: int
    offsets: np.ndarray  # uint32 [n+1]
    cols: np.ndarray  # uint32 [2m]
    labels: np.ndarray  # uint32 [n], 1-based
    edges: np.ndarray  # uint32 [m, 2], each undirected edge once
    name: str = ""

    @property
    def m(self):
        return int(self.edges.shape[0])


@dataclass
class Query:
    labels: np.ndarray  # uint32 [qn]
    edges: np.ndarray  # uint32 [qm, 2] (from, to) in file order
    data_ids: np.ndarray = None  # the walked data vertices (one known match)
    seed: int = 0

    @property
    def n(self):
        return int(self.labels.shape[0])

    @property
    def m(self):
        return int(self.edges.shape[0])


@dataclass
class Workload:
    name: str
    graph: Graph
    queries: list = field(default_factory=list)


def _mix(a, b):
    x = (a * 0x9E3779B97F4A7C15 + b + 0x632BE59BD9B4E019) & 0xFFFFFFFFFFFFFFFF
    x ^= x >> 30
    x = (x * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    x ^= x >> 27
    x = (x * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x ^ (x >> 31)


class Source:
    """Where workloads are drawn: `lib()` returns a ctypes library exporting
    gpsm_gen_er / gpsm_gen_rmat / gpsm_gen_labels / gpsm_gen_query, and
    `csr(n, edges)` returns (offsets, cols)."""

    name = "libgpsm"

    def lib(self):
        return _lib.load()

    def csr(self, n, edges):
        lib = _lib.load()
        m = edges.shape[0]
        off = np.zeros(n + 1, dtype=np.uint32)
        cols = np.zeros(max(2 * m, 1), dtype=np.uint32)
        _lib.check(lib.gpsm_csr_from_edges(n, m, _lib.ptr(edges), _lib.ptr(off), _lib.ptr(cols)), "csr")
        return off, cols[: 2 * m]


ENGINE_SOURCE = Source()


def graph_from_edges(n, edges, labels, name="", source=None):
    source = source or ENGINE_SOURCE
    edges = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 2)
    off, cols = source.csr(n, edges)
    return Graph(n, off, cols, _lib.u32a(labels), edges, name)


def er_graph(n, m, num_labels, seed, zipf_s=0.0, name="er", source=None):
    lib = (source or ENGINE_SOURCE).lib()
    edges = np.zeros((m, 2), dtype=np.uint32)
    _lib.check(lib.gpsm_gen_er(n, m, seed, _lib.ptr(edges)), "gen_er")
    labels = np.zeros(n, dtype=np.uint32)
    _lib.check(lib.gpsm_gen_labels(n, num_labels, zipf_s, _mix(seed, 7), _lib.ptr(labels)), "labels")
    return graph_from_edges(n, edges, labels, name, source)


def rmat_graph(scale, m, num_labels, zipf_s, seed, a=0.57, b=0.19, c=0.19, name="rmat", source=None):
    lib = (source or ENGINE_SOURCE).lib()
    edges = np.zeros((m, 2), dtype=np.uint32)
    _lib.check(lib.gpsm_gen_rmat(scale, m, a, b, c, seed, _lib.ptr(edges)), "gen_rmat")
    n = 1 << scale
    labels = np.zeros(n, dtype=np.uint32)
    _lib.check(lib.gpsm_gen_labels(n, num_labels, zipf_s, _mix(seed, 7), _lib.ptr(labels)), "labels")
    return graph_from_edges(n, edges, labels, name, source)


def random_walk_query(g, qn, seed, mode=MODE_INDUCED, p_extra=0.0, min_avg_degree=0.0, source=None):
    lib = (source or ENGINE_SOURCE).lib()
    ql = np.zeros(qn, dtype=np.uint32)
    qe = np.zeros(max(qn * (qn - 1), 2), dtype=np.uint32)
    ids = np.zeros(qn, dtype=np.uint32)
    r = lib.gpsm_gen_query(g.n, _lib.ptr(g.offsets), _lib.ptr(g.cols), _lib.ptr(g.labels), qn, mode,
                           p_extra, min_avg_degree, seed, _lib.ptr(ql), _lib.ptr(qe), _lib.ptr(ids))
    _lib.check(r, "gen_query")
    return Query(ql, qe[: 2 * r].reshape(-1, 2).copy(), ids, seed)


def _size_stream(rng, kind, count, lo, hi, mean=None):
    if kind == "fixed":
        return [lo] * count
    if kind == "uniform":
        return [int(x) for x in rng.integers(lo, hi + 1, size=count)]
    if kind == "geometric":  # mean `mean`, clipped to [lo, hi]
        p = 1.0 / mean
        return [int(min(hi, max(lo, x))) for x in rng.geometric(p, size=count)]
    raise ValueError(kind)


def query_set(g, count, seed, sizes=("fixed", 6, 6), mix="induced", p_extra=0.3,
              min_avg_degree=0.0, mean=None, source=None, first=0):
    """Queries first .. count-1 of a seeded set of random-walk queries; mix
    is 'induced', 'tree', 'dense' or 'tree_dense' (50/50)."""
    rng = np.random.default_rng(_mix(seed, 0x512E))
    qsizes = _size_stream(rng, sizes[0], count, sizes[1], sizes[2], mean)
    out = []
    for k in range(first, count):
        qs = _mix(seed, 1000 + k)
        if mix == "induced":
            mode = MODE_INDUCED
        elif mix == "tree":
            mode = MODE_TREE
        elif mix == "dense":
            mode = MODE_DENSE
        else:
            mode = MODE_TREE if k % 2 == 0 else MODE_DENSE
        out.append(random_walk_query(g, qsizes[k], qs, mode, p_extra, min_avg_degree, source))
    return out


_GRAPH_CACHE = {}

# name -> (generator, args, seed salt)
_GRAPHS = {
    "small_er": ("er", (10_000, 40_000, 8), 1),
    "rmat20": ("rmat", (20, 16 << 20, 32, 1.0), 2),
    "rmat22": ("rmat", (22, 64 << 20, 64, 1.1), 4),
    "rmat24": ("rmat", (24, 256 << 20, 128, 1.0), 5),
}

# name -> (graph, default count, seed salt, sizes, mix, p_extra, min_avg_degree, mean)
_QUERIES = {
    "small_er": ("small_er", 10, 11, ("fixed", 6, 6), "induced", 0.3, 0.0, None),
    "rmat20": ("rmat20", 100, 12, ("fixed", 12, 12), "induced", 0.3, 2.5, None),
    "rmat20_mix": ("rmat20", 1000, 13, ("uniform", 4, 32), "tree_dense", 0.3, 0.0, None),
    "rmat20_train": ("rmat20", 5000, 14, ("uniform", 4, 32), "tree_dense", 0.3, 0.0, None),
    "rmat22": ("rmat22", 4096, 15, ("uniform", 4, 64), "tree_dense", 0.3, 0.0, None),
    "rmat24": ("rmat24", 2000, 16, ("geometric", 4, 99), "tree_dense", 0.3, 0.0, 16),
}


def graph_for(name, seed=0, source=None):
    source = source or ENGINE_SOURCE
    key = (name, seed, source.name)
    if key in _GRAPH_CACHE:
        return _GRAPH_CACHE[key]
    if name not in _GRAPHS:
        raise ValueError(name)
    kind, args, salt = _GRAPHS[name]
    if kind == "er":
        g = er_graph(*args, _mix(seed, salt), name=name, source=source)
    else:
        g = rmat_graph(*args, _mix(seed, salt), name=name, source=source)
    _GRAPH_CACHE[key] = g
    return g


def workload(name, seed=0, count=None, source=None, first=0):
    """The named workload: graph plus its query set (count overrides the
    size; first > 0 draws only queries first .. first+count-1 of the set,
    the same queries the full set holds at those positions)."""
    if name not in _QUERIES:
        raise ValueError(name)
    gname, default, salt, sizes, mix, p_extra, min_deg, mean = _QUERIES[name]
    g = graph_for(gname, seed, source)
    total = first + (count or default)
    qs = query_set(g, total, _mix(seed, salt), sizes, mix, p_extra, min_deg, mean, source, first=first)
    return Workload(name, g, qs)


def write_text(path, graphs, append=False, terminate=True, first_id=0):
    """Write graphs in the reference's text format (io/IO.cpp:46-128):
    't # id', a count line 'n m vertex_labels edge_labels', 'v i label' per
    vertex, 'e from to 1' per edge; the file ends with 't # -1' (without it
    the reference's reader loops at end of file). Each undirected edge is
    written once. graphs: iterable of (labels, edges)."""
    mode = "a" if append else "w"
    with open(path, mode) as f:
        for k, (labels, edges) in enumerate(graphs):
            labels = np.asarray(labels, np.uint32)
            edges = np.asarray(edges, np.uint32).reshape(-1, 2)
            n, m = len(labels), len(edges)
            f.write(f"t # {first_id + k}\n{n} {m} {len(np.unique(labels))} 1\n")
            if n:
                f.write("\n".join(f"v {i} {int(x)}" for i, x in enumerate(labels)) + "\n")
            if m:
                f.write("\n".join(f"e {int(a)} {int(b)} 1" for a, b in edges) + "\n")
        if terminate:
            f.write("t # -1\n")


def read_text(path):
    """Read every graph of a reference-format text file: [(labels, edges)]."""
    out = []
    labels, edges = None, None
    with open(path) as f:
        for line in f:
            p = line.split()
            if not p:
                continue
            if p[0] == "t":
                if labels is not None:
                    out.append((np.array(labels, np.uint32), np.array(edges, np.uint32).reshape(-1, 2)))
                if int(p[2]) == -1:
                    labels = None
                    break
                labels, edges = [], []
                next(f)  # count line
            elif p[0] == "v":
                labels.append(int(p[2]))
            elif p[0] == "e":
                edges.append((int(p[1]), int(p[2])))
    if labels is not None:
        out.append((np.array(labels, np.uint32), np.array(edges, np.uint32).reshape(-1, 2)))
    return out


def read_text_fast(path):
    """read_text through libgpsm's parallel parser: [(labels, edges)]."""
    import ctypes as C
    lib = _lib.load()
    h = _lib.vp()
    _lib.check(lib.gpsm_text_open(path.encode(), C.byref(h)), "gpsm_text_open")
    try:
        k = C.c_uint32()
        lib.gpsm_text_count(h, C.byref(k))
        out = []
        for i in range(k.value):
            n, m, gid = C.c_uint32(), C.c_uint64(), C.c_int32()
            _lib.check(lib.gpsm_text_graph_info(h, i, C.byref(n), C.byref(m), C.byref(gid)), "gpsm_text_graph_info")
            lab = np.zeros(max(n.value, 1), np.uint32)
            edg = np.zeros((max(m.value, 1), 2), np.uint32)
            _lib.check(lib.gpsm_text_graph_read(h, i, _lib.ptr(lab), _lib.ptr(edg), None), "gpsm_text_graph_read")
            out.append((lab[: n.value], edg[: m.value]))
        return out
    finally:
        lib.gpsm_text_close(h)


def write_text_fast(path, graphs, terminate=True):
    """write_text through libgpsm's buffered writer."""
    lib = _lib.load()
    graphs = list(graphs)
    for k, (labels, edges) in enumerate(graphs):
        lab = _lib.u32a(labels)
        edg = _lib.u32a(np.asarray(edges).reshape(-1))
        _lib.check(lib.gpsm_text_write(path.encode(), 1 if k else 0, k, len(lab), _lib.ptr(lab), len(edg) // 2,
                                       _lib.ptr(edg) if len(edg) else None, None,
                                       1 if (terminate and k == len(graphs) - 1) else 0), "gpsm_text_write")
