"""Join steps that end at a row boundary: with GPSM_DEBUG_WIDE_STEPS=1 every
intermediate step admits 16 times the candidates its output holds rows, so
every step that keeps more than a sixteenth of them keeps more rows than fit
and the write pass ends it at a row boundary (the rest offered again). The
rows must be exactly those of the default steps. Every query here has a work
cap, so a query the plain order handles badly stays bounded."""
import os

import numpy as np
import pytest

from gpsm_b200 import workloads as W

pytestmark = pytest.mark.gpu
WORK = 10**10  # candidates a query's joins may scan: a bound only, these queries finish well within it


def test_steps_cut_at_a_row_boundary_give_the_same_rows(gpu):
    wl = W.workload("rmat20_mix", count=6)
    dg = gpu.DeviceGraph(wl.graph)
    # small levels: many steps per query, so many of them are cut
    ref = [gpu.match(dg, q, cap=100_000, level_bytes=8 << 20, work_cap=WORK) for q in wl.queries]
    assert not any(r.info["aborted"] for r in ref)
    os.environ["GPSM_DEBUG_WIDE_STEPS"] = "1"
    try:
        wide = [gpu.match(dg, q, cap=100_000, level_bytes=8 << 20, work_cap=16 * WORK) for q in wl.queries]
    finally:
        del os.environ["GPSM_DEBUG_WIDE_STEPS"]
    assert not any(o.info["aborted"] for o in wide)
    assert sum(o.info["cut_steps"] for o in wide) > 0
    for r, o in zip(ref, wide):
        assert o.count == r.count
        assert np.array_equal(o.pos2id, r.pos2id)
        assert np.array_equal(o.rows, r.rows)


def test_edge_table_and_list_search_give_the_same_rows(gpu):
    """Steps with more than one placed neighbour check candidates in the
    data graph's edge table; GPSM_DEBUG_NO_EDGE_HASH=1 makes them search the
    candidate-edge lists instead. Dense queries give the same rows either way."""
    wl = W.workload("rmat20_mix", count=6)
    dg = gpu.DeviceGraph(wl.graph)
    slots, probe = dg.edge_table()
    assert slots >= 2 * (len(dg.download()[1]) // 2) and probe < 4096
    dense = [q for q in wl.queries if q.m > q.n - 1]
    assert dense
    with_table = [gpu.match(dg, q, cap=50_000, work_cap=WORK) for q in dense]
    os.environ["GPSM_DEBUG_NO_EDGE_HASH"] = "1"
    try:
        lists = [gpu.match(dg, q, cap=50_000, work_cap=WORK) for q in dense]
    finally:
        del os.environ["GPSM_DEBUG_NO_EDGE_HASH"]
    for a, b in zip(with_table, lists):
        assert a.count == b.count
        assert np.array_equal(a.pos2id, b.pos2id)
        assert np.array_equal(a.rows, b.rows)


_CHILD = """
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import gpsm_b200 as G
from gpsm_b200 import workloads as W
G.init(0)
wl = W.workload("rmat20_mix", count=4)
dg = G.DeviceGraph(wl.graph)
rows = [G.match(dg, q, cap=20_000, work_cap=10**10).rows for q in wl.queries]
np.save(sys.argv[2], np.concatenate([r.ravel() for r in rows]))
"""


def test_blocking_sync_mode_gives_the_same_rows(gpu, tmp_path):
    """GPSM_BLOCKING_SYNC=1 (threads sleep on an event while their stream
    works; read once per process, so a child process runs it) returns the
    same rows as the default waits."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = []
    for mode in ("0", "1"):
        path = str(tmp_path / f"rows{mode}.npy")
        env = dict(os.environ, GPSM_BLOCKING_SYNC=mode)
        subprocess.run([sys.executable, "-c", _CHILD, root, path], env=env, check=True, timeout=600)
        outs.append(np.load(path))
    assert np.array_equal(outs[0], outs[1])
