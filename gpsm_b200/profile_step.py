"""One batch of a workload on the calling thread, for profilers.

    python -m gpsm_b200.profile_step [--workload rmat20] [--first 0] [--count 0]
                                     [--queries 0,2,3] [--order learned|plain]
                                     [--cap 10000000] [--work-cap 0] [--passes 1]

The bench's timed step runs its queries on engine slots (one host thread
and one stream each). This driver runs the same queries, order and cap
through gpsm_match_batch on the default engine instead: one host thread, one
stream, so a kernel profiler sees every launch of the step in order. Set
GPSM_ARENA_GB to keep the workspace small under a profiler. Prints one JSON
line per pass (device ms, launches, join launches, algorithmic join bytes).
"""
import argparse
import json

from . import DeviceGraph, init, match_batch, pack_queries
from . import learned as L
from . import workloads as W


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="rmat20")
    ap.add_argument("--first", type=int, default=0)
    ap.add_argument("--count", type=int, default=0, help="queries from --first (0 = all)")
    ap.add_argument("--order", default="learned", choices=["learned", "plain"])
    ap.add_argument("--cap", type=int, default=10_000_000)
    ap.add_argument("--passes", type=int, default=1)
    ap.add_argument("--queries", default="", help="comma-separated batch indices (instead of --first/--count)")
    ap.add_argument("--work-cap", type=int, default=0, help="candidates a query's joins may scan (0 = none)")
    args = ap.parse_args()
    init(0)
    wl = W.workload(args.workload)
    if args.queries:
        qs = [wl.queries[int(i)] for i in args.queries.split(",")]
    else:
        qs = wl.queries[args.first:]
        if args.count:
            qs = qs[: args.count]
    dg = DeviceGraph(wl.graph)
    model = L.load(0) if args.order == "learned" else None
    packed = pack_queries(qs)
    for p in range(args.passes):
        counts, capped, qms, info = match_batch(dg, qs, cap=args.cap, packed=packed, slots=1,
                                                orders="learned" if model else None, model=model,
                                                work_cap=args.work_cap)
        print(json.dumps({"pass": p, "queries": len(qs), "device_ms": info["device_ms"], "launches": info["launches"],
                          "expand_launches": info["expand_launches"], "alg_bytes_join": info["alg_bytes_join"],
                          "expand_ms": info["expand_ms"], "rows": int(counts.sum())}), flush=True)


if __name__ == "__main__":
    main()
