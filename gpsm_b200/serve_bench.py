"""Serving benchmark: a Poisson request stream against a device-resident graph.

    python -m gpsm_b200.serve_bench [--scale 24] [--rates 200,500,2000] [--requests 1000]
                                    [--slots 8] [--budget-gb 60] [--cap 1000000] [--order learned]
                                    [--work-cap 2000000000] [--slot-arena-gb 16]

Graph: R-MAT(.57,.19,.19,.05) on 2^scale vertices with 16 * 2^scale
undirected edges (2^24: 256 Mi edges, a 2 GiB int32 CSR), labels Zipf(1.0)
over 1..128. Queries: random walks of 4..99 vertices (geometric, mean 16),
half tree, half dense. Requests arrive with exponential gaps at each rate;
the server (gpsm_server_*) admits each request's joins by its predicted
join memory under the budget. A request whose joins reach the work cap
(candidates scanned) stops there and is counted as aborted. Prints one
JSON line per rate: sustained queries/s, embeddings/s and p50/p99 latency
(submit to end, ms).
"""
import argparse
import json
import threading
import time

import numpy as np

from . import DeviceGraph, Server, init
from . import workloads as W


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--rates", default="200,500,2000")
    ap.add_argument("--requests", type=int, default=1000)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--budget-gb", type=float, default=60.0)
    ap.add_argument("--cap", type=int, default=1_000_000)
    ap.add_argument("--order", default="learned", choices=["plain", "learned"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--work-cap", type=int, default=2_000_000_000)
    ap.add_argument("--slot-arena-gb", type=float, default=16.0,
                    help="workspace per slot (filter products, join levels, result buffer)")
    args = ap.parse_args()
    init(0)
    t0 = time.time()
    if args.scale == 24:
        g = W.graph_for("rmat24")
    else:
        g = W.rmat_graph(args.scale, 16 << args.scale, 128, 1.0, seed=W._mix(5, args.scale), name="rmat")
    t_gen = time.time() - t0
    dg = DeviceGraph(g)
    model = None
    if args.order == "learned":
        from . import learned as L
        model = L.load(0)
    qs = W.query_set(g, args.requests, W._mix(args.seed, 16), ("geometric", 4, 99), "tree_dense", 0.3, mean=16)
    budget = int(args.budget_gb * (1 << 30))
    slot_arena = int(args.slot_arena_gb * (1 << 30))
    for rate in [float(r) for r in args.rates.split(",")]:
        srv = Server(dg, slots=args.slots, memory_budget=budget, slot_arena=slot_arena, cap=args.cap,
                     order=args.order, model=model, work_cap=args.work_cap)
        rng = np.random.default_rng(int(rate) + args.seed)
        gaps = rng.exponential(1.0 / rate, size=len(qs))
        tickets = []

        def submitter():
            start = time.perf_counter()
            due = 0.0
            for q, gap in zip(qs, gaps):
                due += gap
                wait = due - (time.perf_counter() - start)
                if wait > 0:
                    time.sleep(wait)
                tickets.append(srv.submit(q))

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        infos = [srv.wait(t, raise_on_error=False) for t in tickets]
        st = srv.stats()
        srv.close()
        ok = [i for i in infos if i["status"] == 0]
        failed = [i for i in infos if i["status"] != 0]
        lat = np.array([i["end_ms"] - i["submit_ms"] for i in ok])
        span_s = (max(i["end_ms"] for i in ok) - min(i["submit_ms"] for i in ok)) / 1e3
        rows = sum(i["rows"] for i in ok)
        print(json.dumps(dict(
            rate_qps=rate, requests=len(qs), completed=len(ok), sustained_qps=len(ok) / span_s,
            embeddings_per_s=rows / span_s, p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
            mean_queue_ms=float(np.mean([i["start_ms"] - i["submit_ms"] for i in ok])),
            peak_admitted_gb=st["peak_in_use"] / 2**30, budget_gb=args.budget_gb, slots=args.slots,
            order=args.order, cap=args.cap, graph=f"rmat 2^{args.scale}, {g.m} edges", graph_gen_s=t_gen,
            capped=int(sum(i["capped"] == 1 for i in ok)), aborted=int(sum(i["capped"] == 2 for i in ok)),
            work_cap=args.work_cap, failed=len(failed),
            first_error=failed[0].get("error") if failed else None)), flush=True)


if __name__ == "__main__":
    main()
