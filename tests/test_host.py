"""Host-side logic: generators, CSR construction, query extraction."""
import numpy as np

from gpsm_b200 import workloads as W


def test_er_is_deterministic_and_simple(lib):
    a = W.er_graph(2000, 6000, 4, seed=5)
    b = W.er_graph(2000, 6000, 4, seed=5)
    assert np.array_equal(a.edges, b.edges) and np.array_equal(a.labels, b.labels)
    e = a.edges.astype(np.int64)
    assert (e[:, 0] < e[:, 1]).all()
    key = e[:, 0] * 2000 + e[:, 1]
    assert len(np.unique(key)) == 6000
    assert a.labels.min() >= 1 and a.labels.max() <= 4


def test_csr_sorted_and_symmetric(lib):
    g = W.er_graph(500, 1500, 3, seed=1)
    off, cols = g.offsets.astype(np.int64), g.cols
    assert off[0] == 0 and off[-1] == 2 * g.m
    for v in range(g.n):
        lst = cols[off[v]:off[v + 1]]
        assert (np.diff(lst.astype(np.int64)) > 0).all()
    pairs = set()
    for v in range(g.n):
        for x in cols[off[v]:off[v + 1]]:
            pairs.add((v, int(x)))
    assert all((b, a) in pairs for a, b in pairs)


def test_rmat_exact_edge_count(lib):
    g = W.rmat_graph(12, 20000, 8, 1.0, seed=3)
    assert g.m == 20000
    e = g.edges.astype(np.int64)
    assert (e[:, 0] != e[:, 1]).all()
    assert len(np.unique(e[:, 0] * 4096 + e[:, 1])) == 20000
    deg = np.diff(g.offsets.astype(np.int64))
    assert deg.max() > 20 * deg.mean()  # skewed


def test_zipf_labels(lib):
    g = W.rmat_graph(14, 30000, 16, 1.0, seed=9)
    cnt = np.bincount(g.labels, minlength=17)[1:]
    assert cnt[0] > cnt[1] > cnt[3] > cnt[15]


def test_random_walk_query_is_connected_and_matches_its_walk(lib):
    g = W.er_graph(3000, 12000, 4, seed=2)
    for s in range(5):
        q = W.random_walk_query(g, 6, s, W.MODE_INDUCED)
        assert q.n == 6 and q.m >= 5
        ids = q.data_ids
        adj = set(map(tuple, g.edges.tolist()))
        for a, b in q.edges:
            x, y = int(ids[a]), int(ids[b])
            assert (min(x, y), max(x, y)) in adj
        assert np.array_equal(q.labels, g.labels[ids])


def test_tree_and_dense_modes(lib):
    g = W.rmat_graph(12, 30000, 4, 1.0, seed=4)
    qt = W.random_walk_query(g, 8, 1, W.MODE_TREE)
    assert qt.m == 7
    qd = W.random_walk_query(g, 8, 1, W.MODE_DENSE, p_extra=1.0)
    qi = W.random_walk_query(g, 8, 1, W.MODE_INDUCED)
    assert qd.m == qi.m


def test_min_average_degree(lib):
    g = W.rmat_graph(14, 60000, 8, 1.0, seed=6)
    q = W.random_walk_query(g, 10, 3, W.MODE_INDUCED, min_avg_degree=2.5)
    assert 2.0 * q.m / q.n >= 2.5
