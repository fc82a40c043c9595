"""Throughput benchmark of the subgraph-matching path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rmat20] [--order learned|plain] [--slots 4] [--cap 10000000]

A step is one pass of the path over one batch of queries against the
device-resident data graph (default: the R-MAT 2^20 workload, 100 induced
random-walk queries of 12 vertices, 10^7-embedding cap per query).

value: queries/s over the K timed steps with the graph and the query batch
already resident, with the learned join order and `--slots` engine slots
(continuous batching); device time from events on the slots' streams, L2
flushed between steps. plain_order: one step of the reference's join order
on one slot (the plain GpSM-order GPU path), for the learned+batched ratio.
e2e: the same metric through the request server (gpsm_server_*), host
buffers in and every embedding row copied back to host memory, all inside
the timed region, after two untimed passes over the same requests (the
library's pool of page-locked result blocks is then grown: steady state).

--impl reference times the CPU port of the reference pipeline (the oracle's
restated filter, refinement, candidate edges and plain-order joins) on all
host cores, on bounded samples of the same workload.

For N > 1 (torchrun) every rank matches its own batch of the same size
against its own replica of the graph (replicas only, weak scaling); the
step time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "queries/s & embeddings/s on 1 B200, learned+batched vs plain order; p50/p99 ms"
WORKLOADS = {
    "rmat20": "R-MAT(.57,.19,.19,.05) 2^20 vertices, 16Mi undirected edges, labels Zipf(1.0) over 1..32; "
              "100 induced random-walk queries of 12 vertices, average degree >= 2.5",
    "small_er": "ER G(10000, 40000), labels U{1..8}; 10 induced random-walk queries of 6 vertices",
    "rmat20_mix": "the rmat20 graph; 1000 tree/dense random-walk queries of 4..32 vertices",
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        if pg.get_backend() == "nccl":
            import torch
            pg.barrier(device_ids=[torch.cuda.current_device()])
        else:
            pg.barrier()


def max_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def load_workload(name, rank, count=None, first=0, take=None):
    wl = _load_workload(name, rank, count)
    if first or take:
        from gpsm_b200 import workloads as W
        qs = wl.queries[first:first + take] if take else wl.queries[first:]
        wl = W.Workload(wl.name, wl.graph, qs)
    return wl


def _load_workload(name, rank, count=None):
    from gpsm_b200 import workloads as W
    wl = W.workload(name, count=count)
    if rank > 0:  # every rank its own batch of the same shape (replicas, weak scaling)
        g = wl.graph
        base = W.workload(name, count=count)
        qs = W.query_set(g, len(base.queries), W._mix(0xB0A7, rank), ("fixed", base.queries[0].n, base.queries[0].n),
                         "induced", min_avg_degree=2.5) if name == "rmat20" else base.queries
        wl = W.Workload(name, g, qs)
    return wl


def cpu_leg(wl, cap, deadline_s, threads=None):
    """The oracle's CPU port on a bounded sample: queries completed per second."""
    import oracle
    threads = threads or os.cpu_count() or 1
    counts, secs = oracle.cpu_pipeline(wl.graph, wl.queries, threads=threads, cap=cap, deadline_s=deadline_s)
    done = int((counts != oracle.DEADLINE_STOPPED).sum())
    return done / max(secs, 1e-9), threads, done, secs


def run_ours(args):
    rank, world, local, pg = dist_setup(args.gpus)
    import gpsm_b200 as G
    G.init(local)
    wl = load_workload(args.workload, rank, first=args.first, take=args.count)
    dg = G.DeviceGraph(wl.graph)
    packed = G.pack_queries(wl.queries)
    nq = len(wl.queries)
    cap = args.cap
    model = None
    if args.order == "learned":
        from gpsm_b200 import learned as L
        model = L.load(local)
    orders = "learned" if args.order == "learned" else None

    def run_step(slots):
        return G.match_batch(dg, wl.queries, cap=cap, packed=packed, slots=slots, orders=orders, model=model)

    # warm-up
    for _ in range(args.warmup):
        run_step(args.slots)
    clocks = ClockSampler(local)
    step_ms, qms_all, launches, rows_total = [], [], 0, 0
    alg_bytes, expand_ms, expand_launches, join_steps = 0, 0.0, 0, 0
    barrier(pg)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        G.flush_l2(256 << 20)
        counts, capped, qms, info = run_step(args.slots)
        step_ms.append(info["device_ms"])
        qms_all.extend(qms.tolist())
        launches += info["launches"]
        rows_total += info["rows"]
        alg_bytes += info["alg_bytes_join"]
        expand_ms += info["expand_ms"]
        expand_launches += info["expand_launches"]
        join_steps += info["join_steps"]
    wall = time.perf_counter() - t0
    barrier(pg)
    clk = clocks.stop()
    dev_s = max_over_ranks(pg, sum(step_ms) / 1e3)
    total_q = sum_over_ranks(pg, nq * args.steps)
    total_rows = sum_over_ranks(pg, rows_total)
    # the plain GpSM-order path (one slot), one step, for the ratio
    plain_ms = None
    if not args.no_plain:
        G.flush_l2(256 << 20)
        pc, _, _, pinfo = G.match_batch(dg, wl.queries, cap=cap, packed=packed, slots=1)
        plain_ms = max_over_ranks(pg, pinfo["device_ms"])
        plain_rows = pinfo["rows"]
    # e2e: the request server with host buffers; rows come back to the host
    h2d = sum(int(q.labels.nbytes + q.edges.nbytes) for q in wl.queries)
    e2e_steps = 1
    barrier(pg)
    srv = G.Server(dg, slots=args.slots, cap=cap, order=args.order if args.order == "learned" else None,
                   model=model, collect_rows=True)
    # two untimed passes: the library's pool of page-locked result blocks
    # grows to what the request stream keeps in flight (steady state)
    for _ in range(2):
        for t in [srv.submit(q) for q in wl.queries]:
            srv.wait(t)
    barrier(pg)
    t1 = time.perf_counter()
    d2h = 0
    for _ in range(e2e_steps):
        tickets = [srv.submit(q) for q in wl.queries]
        for t in tickets:
            r = srv.wait(t)
            d2h += r["table"].nbytes
    e2e_wall = max_over_ranks(pg, time.perf_counter() - t1)
    srv.close()
    d2h //= e2e_steps
    e2e_q = sum_over_ranks(pg, nq * e2e_steps)
    peak, peak_kind = peaks()
    achieved = (alg_bytes / 1e9) / (expand_ms / 1e3) if expand_ms > 0 else 0.0
    result = None
    if rank == 0:
        cpu_rate, cores, done, secs = cpu_leg(wl, cap, args.cpu_seconds) if world == 1 else (None, 0, 0, 0)
        # DRAM bytes per join step (its locate, check, scan and write launches): the
        # ratio of DRAM traffic to algorithmic bytes from one ncu capture of
        # this workload, times this run's algorithmic bytes per step
        traffic = None
        tf = os.path.join(ROOT, "profiles", "expand_traffic.json")
        if os.path.exists(tf) and join_steps:
            ratio = json.load(open(tf)).get("traffic_over_alg")
            if ratio:
                traffic = ratio * alg_bytes / join_steps
        result = {
            "metric": METRIC,
            "value": total_q / dev_s,
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": dev_s * 1e3 / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": args.workload + ": " + WORKLOADS.get(args.workload, ""),
                       "queries_per_step_per_gpu": nq, "embedding_cap": cap, "order": args.order,
                       "slots": args.slots, "l2": "flushed (256 MiB write) between steps",
                       "parallelism": f"replicas x{world}"},
            "plain_order": None if plain_ms is None else {
                "value": total_q / args.steps / (plain_ms / 1e3), "unit": "queries/s", "ms_per_step": plain_ms,
                "slots": 1, "embeddings_per_s": plain_rows / (plain_ms / 1e3)},
            "embeddings_per_s": total_rows / dev_s,
            "p50_ms": float(np.percentile(qms_all, 50)) if qms_all else None,
            "p99_ms": float(np.percentile(qms_all, 99)) if qms_all else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "kernel": "join step (k_locate + k_extend_check + k_scan_u32 + k_extend_write)", "peak_source": peak_kind,
                         "traffic_per": "join step, scaled from profiles/expand_traffic.json",
                         "alg_bytes_per_step": alg_bytes / join_steps if join_steps else None,
                         "join_steps": join_steps,
                         "expand_launches": expand_launches, "expand_ms": expand_ms},
            "cpu_baseline": None if cpu_rate is None else {
                "value": cpu_rate, "unit": "queries/s", "cores": cores, "kind": "port",
                "sample": f"{done} of {nq} queries completed in {secs:.1f} s (deadline {args.cpu_seconds} s), "
                          f"same graph and cap, oracle CPU port on {cores} threads"},
            "e2e": {"value": e2e_q / e2e_wall, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "clocks": clk,
            "wall_s": wall,
        }
        print(json.dumps(result), flush=True)
    dg.free()
    if pg is not None:
        pg.destroy_process_group()
    return result


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    wl = load_workload(args.workload, 0, first=args.first, take=args.count)
    for _ in range(args.warmup):
        pass  # the CPU port has no warm-up state worth priming beyond the first sample
    rates, dones = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rate, cores, done, secs = cpu_leg(wl, args.cap, args.cpu_seconds)
        rates.append(rate)
        dones.append(done)
    wall = time.perf_counter() - t0
    value = float(np.mean(rates))
    result = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "queries/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": wall * 1e3 / max(args.steps, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": args.workload + ": " + WORKLOADS.get(args.workload, ""),
                   "embedding_cap": args.cap, "order": "plain"},
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"each step: queries completed within {args.cpu_seconds} s "
                                   f"({dones} completed per step)"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(result), flush=True)
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat20")
    ap.add_argument("--order", default="learned", choices=["plain", "learned"])
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-order comparison step")
    ap.add_argument("--cap", type=int, default=10_000_000)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--first", type=int, default=0, help="first query of the batch (profiling subsets)")
    ap.add_argument("--count", type=int, default=0, help="queries from --first (0 = all)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
