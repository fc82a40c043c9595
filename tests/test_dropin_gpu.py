"""The reference's own driver loop over this library's drop-in classes.

oracle/ref.mk compiles the reference's unmodified main/run.cpp against
include/gpsm_host/ (Graph, IO, Match) and links it with libgpsm.so. That loop
reads every data graph of a file in turn and deletes each one after its
queries (main/run.cpp:60-98), so the next graph can reuse the deleted one's
address: the drop-in must upload it afresh. The data file here holds two
different graphs; the output must be byte-identical to the reference's own
CUDA build on the same files.

The reference build only runs where its join path is sound: every query must
be a tree (no join_kernel step, whose shared-memory race returns wrong rows
on sm_100a) and its plain order must never pick an edge without a visited
endpoint (match/Match.cu:1639-1650). Both are checked on the CPU with the
oracle's restatement before anything runs.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from gpsm_b200 import workloads as W

pytestmark = pytest.mark.gpu
G = os.path.join(ROOT, "tests", "golden")
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "GpSM.exe")
DROPIN_EXE = os.path.join(ROOT, "oracle", "_ref", "run_dropin")


def _second_graph(n=10_000, m=40_000, seed=77):
    """A seeded ER graph unlike the golden one (numpy only)."""
    rng = np.random.default_rng(seed)
    keys = set()
    while len(keys) < m:
        a, b = rng.integers(0, n, size=2)
        if a != b:
            keys.add((min(a, b), max(a, b)))
    edges = np.array(sorted(keys), np.uint32)
    labels = rng.integers(1, 9, size=n).astype(np.uint32)
    return labels, edges


def _sound_for_reference(graphs, queries):
    for labels, edges in graphs:
        g = oracle.graph_from_edges(len(labels), edges, labels)
        for ql, qe in queries:
            q = oracle.Query(ql, qe)
            if q.m != q.n - 1:
                return False
            p = oracle.RefPlan(g, q)
            if p.status == oracle.REF_OK:
                _, modes, defects = p.steps()
                if (modes == 1).any() or defects.any():
                    return False
    return True


@pytest.mark.skipif(not (os.path.exists(REF_EXE) and os.path.exists(DROPIN_EXE)),
                    reason="reference build absent (oracle/ref.mk)")
def test_reference_driver_over_dropin_two_data_graphs(gpu, tmp_path):
    first = W.read_text(os.path.join(G, "small_er_data.g"))
    graphs = [first[0], _second_graph()]
    queries = W.read_text(os.path.join(G, "small_er_query.g"))
    assert _sound_for_reference(graphs, queries)
    data = tmp_path / "data.g"
    W.write_text(str(data), graphs)
    query = os.path.join(G, "small_er_query.g")
    outs = {}
    for name, exe in (("reference", REF_EXE), ("dropin", DROPIN_EXE)):
        out = tmp_path / f"{name}.txt"
        r = subprocess.run([exe, str(data), query, str(out), "0"], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        assert r.stderr.count("match used:") == 2, r.stderr[-2000:]
        outs[name] = open(out, "rb").read()
    assert outs["dropin"] == outs["reference"]
    # the second graph's embeddings differ from the first's (the test would
    # not see a stale device graph otherwise)
    per_graph = outs["reference"].split(b"query graph:0 ")
    assert len(per_graph) == 3
    rows = [[ln for ln in part.splitlines() if ln.startswith(b"(")] for part in per_graph[1:]]
    assert rows[0] != rows[1]
