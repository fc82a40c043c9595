"""Batched and served matching: same results whatever runs beside them."""
import numpy as np
import pytest

from gpsm_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed(gpu):
    g = W.rmat_graph(14, 120000, 10, 1.0, seed=33)
    qs = [W.random_walk_query(g, 4 + k % 6, 500 + k, W.MODE_DENSE if k % 2 else W.MODE_TREE, 0.4)
          for k in range(24)]
    return g, qs, gpu.DeviceGraph(g)


def test_parallel_batch_equals_sequential(gpu, mixed):
    g, qs, dg = mixed
    c1, k1, _, i1 = gpu.match_batch(dg, qs, cap=200000)
    c4, k4, _, i4 = gpu.match_batch(dg, qs, cap=200000, slots=4)
    assert np.array_equal(c1, c4) and np.array_equal(k1, k4)
    assert i4["rows"] == i1["rows"]


def test_each_result_is_the_same_alone_and_in_the_mix(gpu, mixed):
    g, qs, dg = mixed
    srv = gpu.Server(dg, slots=4, cap=200000, collect_rows=True)
    target = qs[5]
    alone = srv.wait(srv.submit(target))
    tickets = [srv.submit(q) for q in qs]  # 24 queries in flight on 4 slots
    mid = srv.submit(target)
    more = [srv.submit(q) for q in qs[:8]]
    in_mix = srv.wait(mid)
    rest = [srv.wait(t) for t in tickets + more]
    srv.close()
    assert alone["status"] == 0 and in_mix["status"] == 0
    assert alone["rows"] == in_mix["rows"]
    assert np.array_equal(alone["table"][:, alone["id_map"]], in_mix["table"][:, in_mix["id_map"]])
    # and each query in the mix equals its own sequential run
    for q, r in zip(qs, rest[: len(qs)]):
        ref = gpu.match(dg, q, cap=200000)
        assert r["rows"] == ref.count
        assert np.array_equal(r["table"][:, r["id_map"]], ref.embeddings())


def test_admission_keeps_join_memory_within_budget(gpu, mixed):
    g, qs, dg = mixed
    budget = 3 << 30
    srv = gpu.Server(dg, slots=4, memory_budget=budget, cap=100000, slot_arena=2 << 30)
    ts = [srv.submit(q) for q in qs]
    infos = [srv.wait(t) for t in ts]
    st = srv.stats()
    srv.close()
    assert all(i["status"] == 0 for i in infos)
    assert 0 < st["peak_in_use"] <= budget
    assert all(i["admitted_bytes"] > 0 for i in infos if True)
    # latencies are ordered: submit <= start <= admit <= end
    for i in infos:
        assert i["submit_ms"] <= i["start_ms"] <= i["admit_ms"] <= i["end_ms"]


def test_failed_request_reports_the_engine_error(gpu, mixed):
    """A request the engine rejects (a disconnected query) comes back with
    its status and the engine's error text; the other requests are served."""
    g, qs, dg = mixed
    srv = gpu.Server(dg, slots=2, cap=1000, work_cap=10**9)
    bad = W.Query(np.array([1, 1, 1], np.uint32), np.array([[0, 1]], np.uint32))
    tb = srv.submit(bad)
    tg = srv.submit(qs[0])
    info = srv.wait(tb, raise_on_error=False)
    assert info["status"] < 0 and "connected" in info["error"]
    assert srv.wait(tg)["status"] == 0
    with pytest.raises(gpu.GpsmError):
        srv.wait(srv.submit(bad))
    srv.close()


def test_wait_any_returns_every_request_once_in_completion_order(gpu, mixed):
    """Results taken as they finish: every ticket comes back exactly once,
    with the rows of its own query; a request already collected by wait()
    is not returned again; nothing outstanding is an error, not a hang."""
    g, qs, dg = mixed
    srv = gpu.Server(dg, slots=4, cap=200000, collect_rows=True)
    tickets = {srv.submit(q)[0]: q for q in qs}
    first = next(iter(tickets))
    direct = srv.wait((first, tickets[first].n))
    seen = {first}
    ends = []
    for _ in range(len(qs) - 1):
        (tid, qn), r = srv.wait_any()
        assert tid in tickets and tid not in seen and qn == tickets[tid].n
        seen.add(tid)
        ends.append(r["end_ms"])
        ref = gpu.match(dg, tickets[tid], cap=200000)
        assert r["rows"] == ref.count
        assert np.array_equal(r["table"][:, r["id_map"]], ref.embeddings())
    assert seen == set(tickets) and direct["status"] == 0
    assert ends == sorted(ends)  # completion order
    with pytest.raises(gpu.GpsmError):
        srv.wait_any(timeout=0.0)
    srv.close()


def test_rows_copied_while_the_slot_moves_on(gpu, mixed):
    """Small device result buffers (2,000 rows): every capped query flushes
    its rows in many copies through the slot's two persistent buffers, and
    a slot starts its next query while the last copies of the previous one
    still run. Every request's rows equal a sequential match."""
    g, qs, dg = mixed
    # an arena size that is no multiple of anything: the persistent result
    # buffers carved from its top must still start on an aligned address
    srv = gpu.Server(dg, slots=2, cap=50000, collect_rows=True, result_rows=2000, slot_arena=(4 << 30) + 12345)
    tickets = {srv.submit(q)[0]: q for q in qs + qs[:6]}
    for _ in range(len(tickets)):
        (tid, _), r = srv.wait_any()
        ref = gpu.match(dg, tickets[tid], cap=50000)
        assert r["status"] == 0 and r["rows"] == ref.count
        assert np.array_equal(r["table"][:, r["id_map"]], ref.embeddings())
    srv.close()


def test_largest_first_serves_the_biggest_queued_request_next(gpu, mixed):
    """With GPSM_F_LARGEST_FIRST a free slot takes the queued request with
    the most query edges (then vertices): on one slot, every request after
    the first to start ran in non-increasing (edges, vertices) order."""
    g, qs, dg = mixed
    srv = gpu.Server(dg, slots=1, cap=1000, largest_first=True)
    tickets = {srv.submit(q): q for q in qs[:12]}
    infos = {t: srv.wait(t) for t in tickets}
    srv.close()
    started = sorted(tickets, key=lambda t: infos[t]["start_ms"])
    keys = [(tickets[t].m, tickets[t].n) for t in started[1:]]
    assert all(a >= b for a, b in zip(keys, keys[1:])), keys
    assert len(set(keys)) > 1
