"""The oracle pinned on known answers, and its two halves checked against each other.

The reference ships no tests, golden vectors or fixtures (main/test.cpp is an
empty main), so the oracle is pinned here by hand-countable cases, by the
two independent implementations agreeing (backtracking from the definition
vs. the restated reference pipeline), and by the committed fixtures under
tests/golden/ (see test_golden.py).
"""
import itertools

import numpy as np
import pytest

import oracle
from gpsm_b200 import workloads as W


def graph(n, edges, labels):
    # the oracle's own CSR: these tests never run the engine's code
    return oracle.graph_from_edges(n, np.array(edges, np.uint32).reshape(-1, 2), np.array(labels, np.uint32))


def query(labels, edges):
    return W.Query(np.array(labels, np.uint32), np.array(edges, np.uint32).reshape(-1, 2))


def brute_force(g, q):
    """All injective label-preserving maps that keep every query edge."""
    adj = set()
    for a, b in g.edges:
        adj.add((int(a), int(b)))
        adj.add((int(b), int(a)))
    out = []
    for f in itertools.permutations(range(g.n), q.n):
        if any(g.labels[f[i]] != q.labels[i] for i in range(q.n)):
            continue
        if all((f[a], f[b]) in adj for a, b in q.edges):
            out.append(f)
    return sorted(out)


def test_triangle_in_k4(lib):
    g = graph(4, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)], [1, 1, 1, 1])
    q = query([1, 1, 1], [(0, 1), (1, 2), (0, 2)])
    rows, cnt = oracle.enumerate_embeddings(g, q)
    assert cnt == 24  # 4 * 3 * 2 ordered triangles
    assert sorted(map(tuple, rows)) == brute_force(g, q)


def test_labels_restrict(lib):
    g = graph(4, [(0, 1), (1, 2), (2, 3)], [1, 2, 1, 2])
    q = query([1, 2], [(0, 1)])
    rows, cnt = oracle.enumerate_embeddings(g, q)
    # data edges with labels (1,2): (0,1), (2,1), (2,3)
    assert cnt == 3
    assert sorted(map(tuple, rows)) == [(0, 1), (2, 1), (2, 3)]


def test_absent_label_gives_nothing(lib):
    g = graph(3, [(0, 1), (1, 2)], [1, 1, 1])
    q = query([1, 5], [(0, 1)])
    _, cnt = oracle.enumerate_embeddings(g, q)
    assert cnt == 0


@pytest.mark.parametrize("seed", range(6))
def test_random_small_against_brute_force(lib, seed):
    rng = np.random.default_rng(seed)
    n = 9
    pairs = [(a, b) for a in range(n) for b in range(a + 1, n) if rng.random() < 0.4]
    g = graph(n, pairs, rng.integers(1, 3, size=n))
    q = W.random_walk_query(g, 4, 100 + seed, W.MODE_INDUCED)
    rows, cnt = oracle.enumerate_embeddings(g, q)
    assert sorted(map(tuple, rows)) == brute_force(g, q)
    plan = oracle.RefPlan(g, q)
    if plan.status == oracle.REF_OK:
        r2, c2, _, _ = plan.join(injective=True)
        id2pos, _ = plan.mapping()
        assert sorted(map(tuple, r2[:, id2pos])) == sorted(map(tuple, rows))


def test_restatement_agrees_with_backtracking_on_small_er(small_er):
    g = small_er.graph
    for q in small_er.queries:
        rows, cnt = oracle.enumerate_embeddings(g, q)
        plan = oracle.RefPlan(g, q)
        assert plan.status == oracle.REF_OK
        r2, c2, lv, capped = plan.join(injective=True)
        id2pos, pos2id = plan.mapping()
        assert not capped and c2 == cnt
        assert sorted(map(tuple, r2[:, id2pos])) == [tuple(x) for x in rows]
        # the identity walk is always an embedding
        assert tuple(q.data_ids) in set(map(tuple, rows))


def test_reference_table_order_is_lexicographic(small_er):
    """The reference builds its table in column order (seed pairs, then each
    row's new values ascending), so its rows are sorted by table column."""
    g = small_er.graph
    q = small_er.queries[0]
    plan = oracle.RefPlan(g, q)
    r, _, _, _ = plan.join(injective=False)
    keys = [tuple(x) for x in r]
    assert keys == sorted(keys)


def test_homomorphism_table_contains_injective_rows(small_er):
    g = small_er.graph
    q = small_er.queries[1]
    plan = oracle.RefPlan(g, q)
    rh, ch, _, _ = plan.join(injective=False)
    ri, ci, _, _ = plan.join(injective=True)
    inj = [tuple(x) for x in rh if len(set(x.tolist())) == q.n]
    assert inj == [tuple(x) for x in ri]
    assert ch >= ci


def test_parallel_data_edges_give_each_embedding_once(lib):
    g = graph(3, [(0, 1), (0, 1), (1, 2)], [1, 1, 1])
    q = query([1, 1], [(0, 1)])
    rows, cnt = oracle.enumerate_embeddings(g, q)
    assert sorted(map(tuple, rows)) == [(0, 1), (1, 0), (1, 2), (2, 1)]


def test_cap_returns_prefix_in_table_order(small_er):
    g = small_er.graph
    q = small_er.queries[0]
    plan = oracle.RefPlan(g, q)
    full, cnt, _, _ = plan.join(injective=True)
    part, c2, _, capped = plan.join(injective=True, cap=100)
    assert capped and c2 == 100
    assert np.array_equal(part, full[:100])


def test_explore_semantics_skip_after_first_failing_target(lib):
    """explore_kernel (match/Match.cu:528-601) stops at the first target with
    no match, so later targets get no candidates from that data vertex."""
    # query 0(l1)-1(l2), 0(l1)-2(l3); root is 0, targets in order [1, 2].
    # data A=0 (l1): neighbours 1 (l3), 2 (l9) -> no label-2 neighbour;
    #      B=3 (l1): neighbours 4 (l2), 5 (l3).
    g = graph(6, [(0, 1), (0, 2), (3, 4), (3, 5)], [1, 3, 9, 1, 2, 3])
    q = query([1, 2, 3], [(0, 1), (0, 2)])
    plan = oracle.RefPlan(g, q)
    assert list(plan.filter_order()) == [0, 1, 2]
    c = plan.candidates(0)
    assert np.flatnonzero(c[0]).tolist() == [3]  # A cleared
    assert np.flatnonzero(c[1]).tolist() == [4]
    assert np.flatnonzero(c[2]).tolist() == [5]  # not 1: A stopped at target 1


def test_oracle_csr_equals_engine_csr(lib):
    """The oracle's numpy CSR and the engine's gpsm_csr_from_edges agree,
    parallel edges included, so a CSR bug cannot hide on both sides."""
    rng = np.random.default_rng(3)
    for n, m in [(1, 0), (7, 12), (500, 4000), (20_000, 150_000)]:
        e = rng.integers(0, n, size=(m, 2)).astype(np.uint32)
        o = oracle.csr_from_edges(n, e)
        g = W.graph_from_edges(n, e, np.ones(n, np.uint32))
        assert np.array_equal(o[0], g.offsets) and np.array_equal(o[1], g.cols)


@pytest.mark.parametrize("name", ["small_er", "rmat20_mix"])
def test_oracle_source_draws_the_engine_workloads(lib, name):
    """Workloads drawn without libgpsm.so (what bench.py's reference arm
    uses) are the ones the engine's source draws: same graph, CSR and
    queries; a window [first, first+count) equals that slice of the set."""
    if name == "rmat20_mix":  # the graph shape at a size the CPU suite affords
        W._GRAPHS["_t14"] = ("rmat", (14, 1 << 17, 16, 1.0), 9)
        W._QUERIES["_t14_mix"] = ("_t14", 30, 13, ("uniform", 4, 32), "tree_dense", 0.3, 0.0, None)
        name = "_t14_mix"
    a = W.workload(name)
    b = W.workload(name, source=oracle.GEN_SOURCE)
    for x, y in [(a.graph.offsets, b.graph.offsets), (a.graph.cols, b.graph.cols),
                 (a.graph.labels, b.graph.labels), (a.graph.edges, b.graph.edges)]:
        assert np.array_equal(x, y)
    assert len(a.queries) == len(b.queries)
    for qa, qb in zip(a.queries, b.queries):
        assert np.array_equal(qa.labels, qb.labels) and np.array_equal(qa.edges, qb.edges)
    w = W.workload(name, first=3, count=4, source=oracle.GEN_SOURCE)
    for qa, qb in zip(a.queries[3:7], w.queries):
        assert np.array_equal(qa.labels, qb.labels) and np.array_equal(qa.edges, qb.edges)
