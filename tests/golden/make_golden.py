"""Generate the golden fixtures that pin the oracle to the reference itself.

The reference has no tests or golden vectors, so this script runs the
reference's own build (oracle/_ref/ref_driver, compiled from the unmodified
sources by oracle/ref.mk) on seeded inputs and stores its raw result tables
(the Match::match output before io/IO.cpp's directed/label filter).

  python tests/golden/make_golden.py inputs   # write the .g input files (CPU)
  python tests/golden/make_golden.py run      # run the reference (needs a GPU)
  python tests/golden/make_golden.py pack     # .bin -> golden .npz (table prefixes + row counts)

Only queries for which the restated reference (oracle.RefPlan) shows a
well-defined run are kept: no expand pick with an unvisited endpoint pair
(match/Match.cu:1639-1650, which would read column -1) and homomorphism
tables small enough that the reference's 32-bit grid arithmetic cannot
overflow (match/Match.cu:1313, 1515).
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SETS = ["small_er", "rmat12"]
MAX_TABLE_ROWS = 1 << 20
PREFIX_ROWS = 40000  # rows kept per table (tables are in a fixed order); the full count is kept too


def build_set(name):
    from gpsm_b200 import workloads as W
    if name == "small_er":
        wl = W.workload("small_er")
        return wl.graph, wl.queries
    if name == "rmat12":
        g = W.rmat_graph(12, 20000, 12, 1.0, seed=W._mix(7, 12), name="rmat12")
        qs = []
        k = 0
        while len(qs) < 12:
            mode = [W.MODE_INDUCED, W.MODE_DENSE, W.MODE_TREE][k % 3]
            q = W.random_walk_query(g, 4 + (k % 4), W._mix(70, k), mode, 0.5)
            k += 1
            if safe(g, q):
                qs.append(q)
        return g, qs
    raise ValueError(name)


def safe(g, q):
    import oracle
    plan = oracle.RefPlan(g, q)
    if plan.status not in (oracle.REF_OK, oracle.REF_EMPTY_INIT, oracle.REF_EMPTY_REFINE):
        return False
    if plan.defect:
        return False
    if plan.status == oracle.REF_OK:
        _, cnt, lv, capped = plan.join(injective=False, rows=False, cap=MAX_TABLE_ROWS,
                                       work_cap=8 * MAX_TABLE_ROWS)
        if capped or int(lv.max()) >= MAX_TABLE_ROWS:
            return False
    return True


def paths(name):
    return (os.path.join(HERE, f"{name}_data.g"), os.path.join(HERE, f"{name}_query.g"),
            os.path.join(HERE, f"{name}_ref.bin"), os.path.join(HERE, f"{name}_ref.npz"))


def inputs():
    from gpsm_b200 import workloads as W
    for name in SETS:
        g, qs = build_set(name)
        for q in qs:
            assert safe(g, q), name
        d, qp, _, _ = paths(name)
        W.write_text(d, [(g.labels, g.edges)])
        W.write_text(qp, [(q.labels, q.edges) for q in qs])
        print(name, g.n, g.m, len(qs))


def run():
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    for name in SETS:
        d, qp, b, _ = paths(name)
        with open(b + ".log", "w") as log:
            subprocess.run([drv, d, qp, b, "0"], check=True, stdout=log, stderr=subprocess.STDOUT)


def read_bin(path):
    recs = []
    raw = open(path, "rb").read()
    off = 0
    while off < len(raw):
        qid, rows, cols = np.frombuffer(raw, np.int32, 1, off)[0], *np.frombuffer(raw, np.uint32, 2, off + 4)
        ms = np.frombuffer(raw, np.float32, 1, off + 12)[0]
        off += 16
        idm = np.frombuffer(raw, np.int32, cols, off).copy()
        off += 4 * cols
        tab = np.frombuffer(raw, np.uint32, int(rows) * int(cols), off).copy().reshape(int(rows), int(cols))
        off += 4 * int(rows) * int(cols)
        recs.append((int(qid), idm, tab, float(ms)))
    return recs


def pack():
    for name in SETS:
        _, _, b, z = paths(name)
        recs = read_bin(b)
        arrays = {}
        for qid, idm, tab, ms in recs:
            arrays[f"q{qid}_id_map"] = idm
            arrays[f"q{qid}_table"] = tab[:PREFIX_ROWS]
            arrays[f"q{qid}_rows"] = np.array(tab.shape[0], np.int64)
            arrays[f"q{qid}_ms"] = np.array(ms, np.float32)
        arrays["n_queries"] = np.array(len(recs))
        np.savez_compressed(z, **arrays)
        print(name, len(recs), "queries", sum(t.shape[0] for _, _, t, _ in recs), "rows")


if __name__ == "__main__":
    {"inputs": inputs, "run": run, "pack": pack}[sys.argv[1]]()

# small_er_ans.txt is the output file of the reference's own command line
# driver (oracle/_ref/GpSM.exe, main/run.cpp) on small_er_{data,query}.g:
#   oracle/_ref/GpSM.exe tests/golden/small_er_data.g tests/golden/small_er_query.g small_er_ans.txt 0
# (rows after io/IO.cpp's directed, edge-labelled verify, in table order).
