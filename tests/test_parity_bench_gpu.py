"""Parity on the benchmarked workloads, against the backtracking oracle.

The engine emits a match in one vertex order (the plain order, a learned
plan, or whichever of the two finishes first when they race) and its rows
come out in the lexicographic order of their values taken in that order; a
cap keeps the first `cap` of them. oracle.enumerate_ordered searches the
same order from the definition of an embedding (it shares no code with the
engine and reads the oracle's own CSR), so for every query here:
  - at cap 10^5: the engine's rows equal the oracle's first 10^5 rows in the
    engine's finishing order, row for row;
  - at cap 10^7 (the benchmark's cap): the counts are equal and the
    order-sensitive digests of all rows are equal.
Queries come from the benchmark's own batches: the R-MAT 2^22 batch of 4,096
uneven queries, the R-MAT 2^20 batch of 100 queries of 12 vertices and the
mixed 4..32-vertex set on the same graph. The oracle must finish every query
here within its work bound: a bound that hides a query fails the test.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

import oracle
from gpsm_b200 import workloads as W

pytestmark = pytest.mark.gpu
WORK = 2 * 10**10  # oracle search steps per query (a query that needs more fails the test)
RMAT22_IDX = [0, 3, 5, 410, 821, 1230, 1641, 2050, 2461, 2870]


@pytest.fixture(scope="module")
def model(gpu):
    from gpsm_b200 import learned as L
    return L.load(0)


def _oracle(g, jobs, cap, rows):
    """enumerate_ordered over (query, pos2id) jobs on all host threads."""
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        futs = [ex.submit(oracle.enumerate_ordered, g, q, list(order), cap, WORK, rows, True) for q, order in jobs]
        return [f.result() for f in futs]


def _rows_vs_oracle(gpu, dg, og, queries, model, cap, order="learned"):
    outs = [gpu.match(dg, q, cap=cap, order=order, model=model) for q in queries]
    refs = _oracle(og, [(q, o.pos2id) for q, o in zip(queries, outs)], cap, True)
    for k, (o, (rows, cnt, _)) in enumerate(zip(outs, refs)):
        assert o.count == cnt, (k, o.count, cnt)
        assert np.array_equal(o.rows, rows), k
    return outs


def _digests_vs_oracle(gpu, dg, og, queries, model, cap):
    got = []
    for q in queries:  # one query's rows in host memory at a time
        o = gpu.match(dg, q, cap=cap, order="learned", model=model)
        got.append((o.count, oracle.rows_digest(o.rows), list(o.pos2id)))
        del o
    refs = _oracle(og, [(q, g[2]) for q, g in zip(queries, got)], cap, False)
    for k, ((cnt, dig, _), (_, rcnt, rdig)) in enumerate(zip(got, refs)):
        assert cnt == rcnt, (k, cnt, rcnt)
        assert dig == rdig, k


@pytest.fixture(scope="module")
def rmat22(gpu):
    wl = W.workload("rmat22", count=max(RMAT22_IDX) + 1)
    og = W.workload("rmat22", count=1, source=oracle.GEN_SOURCE).graph  # the oracle's own CSR
    return wl, gpu.DeviceGraph(wl.graph), og


@pytest.fixture(scope="module")
def rmat20(gpu):
    wl = W.workload("rmat20")
    og = W.workload("rmat20", count=1, source=oracle.GEN_SOURCE).graph
    return wl, gpu.DeviceGraph(wl.graph), og


def test_rmat22_batch_rows_at_cap_1e5(gpu, rmat22, model):
    """Ten queries of the 4,096-query batch (tree and dense, 8..60
    vertices): learned order and plain order, first 10^5 rows."""
    wl, dg, og = rmat22
    qs = [wl.queries[i] for i in RMAT22_IDX]
    outs = _rows_vs_oracle(gpu, dg, og, qs, model, 100_000)
    assert all(o.count == 100_000 for o in outs)
    tree = [q for q in qs if q.m == q.n - 1]
    _rows_vs_oracle(gpu, dg, og, tree, None, 100_000, order=None)


def test_rmat22_batch_digests_at_bench_cap(gpu, rmat22, model):
    """Six of them (tree and dense) at the benchmark's cap of 10^7 rows:
    count and digest of every row."""
    wl, dg, og = rmat22
    _digests_vs_oracle(gpu, dg, og, [wl.queries[i] for i in (0, 3, 410, 821, 1230, 2461)], model, 10_000_000)


def test_rmat20_bench_rows_at_cap_1e5(gpu, rmat20, model):
    """The first 20 queries of the 100-query batch in the learned (raced)
    order, first 10^5 rows."""
    wl, dg, og = rmat20
    _rows_vs_oracle(gpu, dg, og, wl.queries[:20], model, 100_000)


def test_rmat20_bench_counts_and_digests_at_cap_1e7(gpu, rmat20, model):
    """All 100 queries of the batch through the batched entry point (the
    benchmark's call): counts at cap 10^7 equal the oracle's; ten queries
    spread over the batch also by the digest of all their rows."""
    wl, dg, og = rmat20
    counts, _, _, info = gpu.match_batch(dg, wl.queries, cap=10_000_000, slots=4, orders="learned", model=model)
    assert info["aborted"] == 0
    orders = [gpu.match(dg, q, cap=100, order="learned", model=model).pos2id for q in wl.queries]
    refs = _oracle(og, list(zip(wl.queries, orders)), 10_000_000, False)
    assert [int(c) for c in counts] == [cnt for _, cnt, _ in refs]
    _digests_vs_oracle(gpu, dg, og, wl.queries[::10], model, 10_000_000)


def test_rmat20_mix_rows_at_cap_1e5(gpu, rmat20, model):
    """Ten queries of the mixed set (4..32 vertices, tree and dense) on the
    same graph, learned order, first 10^5 rows."""
    _, dg, og = rmat20
    qs = W.workload("rmat20_mix", count=10).queries
    _rows_vs_oracle(gpu, dg, og, qs, model, 100_000)
