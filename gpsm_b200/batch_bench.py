"""Batch benchmark: many uneven queries against one device-resident graph.

    python -m gpsm_b200.batch_bench [--scale 22] [--queries 4096] [--slots 0]
                                    [--cap 10000000] [--work-cap 5000000000]

Graph: R-MAT(.57,.19,.19,.05), 2^22 vertices, 64 Mi undirected edges,
labels Zipf(1.1) over 1..64. Queries: 4,096 random walks of 4..64 vertices
(half tree, half dense). Two arms over the same batch:
  learned+batched  learned join order, `slots` engine slots (0 = tuning)
  plain            the reference's join order, one slot, one query at a time
Both arms use the same embedding cap and the same work cap (candidates a
query's joins may scan; a query that reaches it stops and is counted as
"aborted"). Prints one JSON line per arm and the ratio.
"""
import argparse
import json
import time

import numpy as np

from . import DeviceGraph, get_tuning, init, match_batch
from . import learned as L
from . import workloads as W


def arm(dg, qs, cap, work_cap, slots, order, model):
    import ctypes as C

    from . import _lib
    lib = _lib.load()
    voff, ql, eoff, qe = __import__("gpsm_b200").pack_queries(qs)
    opts = _lib.MatchOpts()
    opts.cap = cap
    opts.work_cap = work_cap
    if order == "learned":
        opts.order_mode = _lib.GPSM_ORDER_LEARNED
        opts.model = model.handle
    n = len(qs)
    counts = np.zeros(n, np.uint64)
    capped = np.zeros(n, np.int32)
    qms = np.zeros(n, np.float64)
    info = _lib.BatchInfo()
    t0 = time.perf_counter()
    rc = lib.gpsm_match_batch_parallel(dg.handle, n, _lib.ptr(voff), _lib.ptr(ql), _lib.ptr(eoff), _lib.ptr(qe),
                                       C.byref(opts), None, slots, 0, _lib.ptr(counts), _lib.ptr(capped),
                                       _lib.ptr(qms), C.byref(info))
    wall = time.perf_counter() - t0
    _lib.check(rc, "gpsm_match_batch_parallel")
    dev_s = info.device_ms / 1e3
    return dict(order=order, slots=slots, queries=n, device_s=dev_s, wall_s=wall, queries_per_s=n / dev_s,
                embeddings_per_s=float(counts.sum()) / dev_s, p50_ms=float(np.percentile(qms, 50)),
                p99_ms=float(np.percentile(qms, 99)), capped=int((capped == 1).sum()),
                aborted=int((capped == 2).sum()), counts=counts)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--queries", type=int, default=4096)
    ap.add_argument("--slots", type=int, default=0)
    ap.add_argument("--cap", type=int, default=10_000_000)
    ap.add_argument("--work-cap", type=int, default=5_000_000_000)
    ap.add_argument("--skip-plain", action="store_true")
    args = ap.parse_args()
    init(0)
    slots = args.slots or get_tuning()["slots"]
    t0 = time.time()
    wl = W.workload("rmat22" if args.scale == 22 else "rmat20_mix", count=args.queries)
    t_gen = time.time() - t0
    dg = DeviceGraph(wl.graph)
    model = L.load(0)
    warm = wl.queries[: min(64, len(wl.queries))]
    match_batch(dg, warm, cap=args.cap, slots=slots, orders="learned", model=model)
    res = {}
    res["learned"] = arm(dg, wl.queries, args.cap, args.work_cap, slots, "learned", model)
    if not args.skip_plain:
        res["plain"] = arm(dg, wl.queries, args.cap, args.work_cap, 1, "plain", None)
    for k, r in res.items():
        print(json.dumps({**{a: b for a, b in r.items() if a != "counts"}, "graph_gen_s": t_gen,
                          "graph": f"rmat 2^{args.scale}", "cap": args.cap, "work_cap": args.work_cap}), flush=True)
    if "plain" in res:
        a, b = res["learned"], res["plain"]
        same = int(np.sum(a["counts"] == b["counts"]))
        print(json.dumps(dict(learned_batched_over_plain=a["queries_per_s"] / b["queries_per_s"],
                              queries_with_equal_counts=same, queries=len(wl.queries))), flush=True)


if __name__ == "__main__":
    main()
