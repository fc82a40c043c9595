"""Throughput benchmark of the subgraph-matching path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rmat22|rmat20|small_er] [--slots 0] [--cap 10000000]

Default workload (the batched uneven-query configuration): R-MAT(.57,.19,
.19,.05) with 2^22 vertices and 64 Mi undirected edges, labels Zipf(1.1) over
1..64, 4,096 random-walk queries of 4..64 vertices (half tree, half dense),
an embedding cap of 10^7 rows per query and a work cap of 5*10^9 candidates
scanned per query (a query that reaches it stops and is counted as
aborted; both orders run under the same caps). The batch is cut into 20
fixed slices of ~205 queries: step k matches slice k mod 20, so 20 timed
steps cover the whole batch once.

value: queries/s over the K timed steps, graph and queries resident in HBM,
with the learned join order on `--slots` engine slots (continuous batching;
0 = the tuned count); device time from events on the slots' streams (span of
the step), L2 flushed (256 MiB write) before every step.
plain_order: the reference's join order on one slot over every fifth slice
(0, 5, 10, 15), with the learned+batched device time of the same slices
beside it.
e2e: the same metric through the request server (gpsm_server_*): query
arrays from host memory and every embedding row copied back to host memory,
inside the timed region, over slice 0 after one untimed pass.
cpu_baseline: the oracle's CPU port of the reference pipeline (filter,
refinement, candidate edges, plain-order joins with injectivity) on all host
threads over a fixed sample (the first 32 queries of the batch with at most
8 vertices); the GPU arm's time on exactly that sample is reported beside it.
reference_build: the reference's own CUDA build (oracle/_ref/GpSM.exe, built
from its unmodified sources) and this library's gpsm_run through the same
run.cpp loop on the small ER set (10 tree queries repeated 20 times).

--impl reference times the CPU port (the reference has no CPU
implementation of the path) on the same fixed sample per step, drawing the
workload without loading libgpsm.so.

For N > 1 (torchrun) every rank matches its own slices against its own
replica of the graph (replicas only, weak scaling): at step k rank r takes
slice (k*N + r) mod 20; the step time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "queries/s & embeddings/s on 1 B200, learned+batched vs plain order; p50/p99 ms"
# name -> description, slices per batch, embedding cap, work cap, plain-order slices, CPU sample rule
WORKLOADS = {
    "rmat22": dict(
        desc="R-MAT(.57,.19,.19,.05) 2^22 vertices, 64Mi undirected edges, labels Zipf(1.1) over 1..64; "
             "4096 random-walk queries of 4..64 vertices (half tree, half dense with extra induced edges at "
             "p=0.3); embedding cap 10^7 per query, work cap 5e9 candidates per query; 20 fixed slices of "
             "~205 queries, step k = slice k mod 20",
        slices=20, cap=10_000_000, work_cap=5_000_000_000, plain=[0, 5, 10, 15], cpu=(8, 32)),
    "rmat20": dict(
        desc="R-MAT(.57,.19,.19,.05) 2^20 vertices, 16Mi undirected edges, labels Zipf(1.0) over 1..32; 100 "
             "induced random-walk queries of 12 vertices, average degree >= 2.5; embedding cap 10^7 per query; "
             "step = the whole batch",
        slices=1, cap=10_000_000, work_cap=0, plain=[0], cpu=(12, 16)),
    "small_er": dict(
        desc="ER G(10000, 40000), labels U{1..8}; 10 induced random-walk queries of 6 vertices; no cap; "
             "step = the whole batch",
        slices=1, cap=0, work_cap=0, plain=[0], cpu=(6, 10)),
}
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "GpSM.exe")
OUR_CLI = os.path.join(ROOT, "gpsm_b200", "gpsm_run")
GOLDEN = os.path.join(ROOT, "tests", "golden")


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


def dist_setup():
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


def _reduce(pg, x, op):
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=op(pg))
    return float(t.item())


def max_over_ranks(pg, x):
    return _reduce(pg, x, lambda d: d.ReduceOp.MAX)


def sum_over_ranks(pg, x):
    return _reduce(pg, x, lambda d: d.ReduceOp.SUM)


def slice_bounds(nq, nslices):
    return [(nq * s // nslices, nq * (s + 1) // nslices) for s in range(nslices)]


def slice_of(k, rank, world, nslices):
    """The slice rank `rank` of `world` matches at step k: the ranks of one
    step take consecutive slices, so each rank does one slice's work."""
    return (k * world + rank) % nslices


def cpu_sample(queries, rule):
    """The fixed CPU sample: the first `count` queries of the batch with at
    most `max_n` vertices (indices into the batch)."""
    max_n, count = rule
    return [i for i, q in enumerate(queries) if q.n <= max_n][:count]


def config_of(args, spec, nq_step, world):
    """The workload description; the same dict on both arms."""
    return {"workload": args.workload + ": " + spec["desc"], "queries_per_step_per_gpu": nq_step,
            "embedding_cap": spec["cap"], "work_cap_candidates": spec["work_cap"],
            "l2": "flushed (256 MiB write) before every step; the CSR alone exceeds L2 on rmat20/rmat22",
            "parallelism": f"replicas x{world}"}


def cpu_leg(graph, queries, cap, threads=None):
    """The oracle's CPU port over `queries` on `threads` host threads:
    (queries/s, threads, seconds, counts)."""
    import oracle
    threads = threads or os.cpu_count() or 1
    counts, secs = oracle.cpu_pipeline(graph, queries, threads=threads, cap=cap or (1 << 62))
    return len(queries) / max(secs, 1e-9), threads, secs, counts


def _match_ms(stderr):
    import re
    m = re.findall(r"match used:\s*(\d+)\s*ms", stderr)
    return sum(int(x) for x in m) if m else None


def reference_build_leg(repeat=20):
    """The reference's own CUDA build and gpsm_run on the small ER set
    (10 tree queries repeated `repeat` times) through the same run.cpp loop:
    per query Match::match, IO::output (host verify + text), flush. Both must
    write the same file."""
    if not (os.path.exists(REF_EXE) and os.path.exists(OUR_CLI)):
        return {"unavailable": "reference build or gpsm_run not built"}
    blocks, cur = [], None
    for line in open(os.path.join(GOLDEN, "small_er_query.g")):
        if line.startswith("t #"):
            if line.split()[2] == "-1":
                break
            cur = []
            blocks.append(cur)
        elif cur is not None:
            cur.append(line)
    with tempfile.TemporaryDirectory() as d:
        qf = os.path.join(d, "q.g")
        with open(qf, "w") as f:
            k = 0
            for _ in range(repeat):
                for b in blocks:
                    f.write(f"t # {k}\n")
                    f.writelines(b)
                    k += 1
            f.write("t # -1\n")
        res = {}
        for name, exe in (("reference", REF_EXE), ("ours", OUR_CLI)):
            out = os.path.join(d, name + ".txt")
            r = subprocess.run([exe, os.path.join(GOLDEN, "small_er_data.g"), qf, out, "0"], capture_output=True,
                               text=True, timeout=600)
            if r.returncode != 0:
                return {"unavailable": f"{name} exited {r.returncode}"}
            res[name] = (_match_ms(r.stderr), open(out, "rb").read())
    (t_ref, a_ref), (t_our, a_our) = res["reference"], res["ours"]
    return {"workload": f"small_er: 10 tree queries of 6 vertices x{repeat}, main/run.cpp loop (Match::match + "
                        "IO::output + flush per query), 'match used' wall time",
            "queries": k, "reference_ms": t_ref, "ours_ms": t_our,
            "reference_qps": k / max(t_ref, 1) * 1e3, "ours_qps": k / max(t_our, 1) * 1e3,
            "identical_output": a_ref == a_our,
            "reference_exe": "oracle/_ref/GpSM.exe (unmodified reference sources, nvcc -O2 sm_100a)",
            "ours_exe": "gpsm_b200/gpsm_run"}


def rank_host_settings(local_world, environ, ram_gb):
    """Environment a rank sets before the library starts when `local_world`
    ranks share this host: every rank is a process with its own pool of
    page-locked result blocks (default: a quarter of host memory each), so
    they share that quarter unless the caller chose a size; and their slot
    threads share the host's cores, so they sleep while their GPU works
    instead of spinning."""
    out = {}
    if local_world > 1:
        if "GPSM_HOST_POOL_GB" not in environ:
            out["GPSM_HOST_POOL_GB"] = str(max(2.0, min(64.0, ram_gb / 4) / local_world))
        if "GPSM_BLOCKING_SYNC" not in environ:
            out["GPSM_BLOCKING_SYNC"] = "1"
    return out


def run_ours(args):
    rank, world, local, pg = dist_setup()
    local_world = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
    ram_gb = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 2**30
    os.environ.update(rank_host_settings(local_world, os.environ, ram_gb))
    import gpsm_b200 as G
    from gpsm_b200 import workloads as W
    G.init(local)
    spec = WORKLOADS[args.workload]
    wl = W.workload(args.workload)
    dg = G.DeviceGraph(wl.graph)
    slots = args.slots or G.get_tuning()["slots"]
    cap = args.cap if args.cap is not None else spec["cap"]
    work_cap = spec["work_cap"]
    model = None
    if args.order == "learned":
        from gpsm_b200 import learned as L
        model = L.load(local)
    orders = "learned" if args.order == "learned" else None
    nq = len(wl.queries)
    bounds = slice_bounds(nq, spec["slices"])
    packs = [G.pack_queries(wl.queries[a:b]) for a, b in bounds]

    def run_slice(s, order, nslots, mdl):
        a, b = bounds[s]
        return G.match_batch(dg, wl.queries[a:b], cap=cap, packed=packs[s], slots=nslots, orders=order, model=mdl,
                             work_cap=work_cap)

    for k in range(args.warmup):
        run_slice(slice_of(k, rank, world, len(bounds)), orders, slots, model)
    clocks = ClockSampler(local)
    step_ms, slice_ms, qms_all, aborted = [], {}, [], 0
    tot = dict(launches=0, rows=0, alg_bytes_join=0, expand_ms=0.0, join_steps=0, queries=0)
    barrier(pg)
    clocks.start()
    t0 = time.perf_counter()
    for k in range(args.steps):
        s = slice_of(k, rank, world, len(bounds))
        G.flush_l2(256 << 20)
        counts, capped, qms, info = run_slice(s, orders, slots, model)
        step_ms.append(info["device_ms"])
        slice_ms[s] = info["device_ms"]
        qms_all.extend(qms.tolist())
        aborted += int(info.get("aborted", 0))
        tot["queries"] += len(counts)
        for key in ("launches", "rows", "alg_bytes_join", "expand_ms", "join_steps"):
            tot[key] += info[key]
    wall = time.perf_counter() - t0
    barrier(pg)
    clk = clocks.stop()
    dev_s = max_over_ranks(pg, sum(step_ms) / 1e3)
    total_q = sum_over_ranks(pg, tot["queries"])
    total_rows = sum_over_ranks(pg, tot["rows"])
    alg_bytes = sum_over_ranks(pg, tot["alg_bytes_join"])

    # the plain GpSM-order path on one slot over fixed slices, against the
    # learned+batched time of the same slices (N = 1 only)
    plain = None
    if world == 1 and not args.no_plain:
        ps = [s for s in spec["plain"] if s in slice_ms]
        if ps:
            p_ms, p_q, p_rows, p_ab, p_exp, p_abort = 0.0, 0, 0, 0, 0.0, 0
            for s in ps:
                G.flush_l2(256 << 20)
                pc, _, _, pinfo = run_slice(s, None, 1, None)
                p_ms += pinfo["device_ms"]
                p_q += len(pc)
                p_rows += pinfo["rows"]
                p_ab += pinfo["alg_bytes_join"]
                p_exp += pinfo["expand_ms"]
                p_abort += int(pinfo.get("aborted", 0))
            l_ms = sum(slice_ms[s] for s in ps)
            plain = {"slices": ps, "queries": p_q, "slots": 1, "order": "plain (reference heuristic)",
                     "value": p_q / (p_ms / 1e3), "unit": "queries/s", "device_ms": p_ms,
                     "embeddings_per_s": p_rows / (p_ms / 1e3), "aborted_at_work_cap": p_abort,
                     "learned_batched_same_slices": {"value": p_q / (l_ms / 1e3), "device_ms": l_ms,
                                                     "slots": slots},
                     "join_one_slot": {"achieved_gbs": (p_ab / 1e9) / (p_exp / 1e3) if p_exp else None,
                                       "note": "algorithmic join bytes / summed join-step event time; one slot, "
                                               "so the events do not overlap"}}

    # e2e: the request server from host buffers, every row back to host memory
    e2e_slices = [slice_of(0, rank, world, len(bounds))]
    e2e_qs = [q for s in e2e_slices for q in wl.queries[bounds[s][0]:bounds[s][1]]]
    h2d = sum(int(q.labels.nbytes + q.edges.nbytes) for q in e2e_qs)
    barrier(pg)
    # the batch slots and the one-slot plain leg keep their arenas: the
    # server's slots share most of what is left. A failure here is reported
    # in the line (every rank still takes the same collective steps).
    import torch
    free_b, _ = torch.cuda.mem_get_info(local)
    e2e_err, srv = None, None
    d2h, e2e_rows = 0, 0
    # the leg is bound by the rows' copy to the host: at most 8 server slots,
    # each with room for the largest queries' joins next to its result buffers
    e2e_slots = min(slots, 8)
    try:
        srv = G.Server(dg, slots=e2e_slots, cap=cap, order=args.order if args.order == "learned" else None,
                       model=model, collect_rows=True, work_cap=work_cap,
                       slot_arena=min(12 << 30, int(0.8 * free_b / e2e_slots)) >> 21 << 21, largest_first=True)
        for q in e2e_qs:  # untimed: grows the pool of page-locked result blocks
            srv.submit(q)
        for _ in e2e_qs:
            srv.wait_any()
    except G.GpsmError as ex:
        e2e_err = str(ex)
    barrier(pg)
    pool0 = G.host_pool_stats()
    t1 = time.perf_counter()
    if e2e_err is None:
        try:
            for q in e2e_qs:
                srv.submit(q)
            for _ in e2e_qs:  # results as they finish, so host memory holds only what is still running
                _, r = srv.wait_any()
                d2h += r["table"].nbytes
                e2e_rows += int(r["rows"])
                del r
        except G.GpsmError as ex:
            e2e_err = str(ex)
    e2e_wall = max_over_ranks(pg, time.perf_counter() - t1)
    pool1 = G.host_pool_stats()
    if srv is not None:
        try:
            srv.close()
        except G.GpsmError:
            pass
    e2e_failed = max_over_ranks(pg, 1.0 if e2e_err else 0.0) > 0
    e2e_q = sum_over_ranks(pg, len(e2e_qs))
    e2e_d2h = sum_over_ranks(pg, d2h)

    peak, peak_kind = peaks()
    achieved = (alg_bytes / 1e9) / dev_s if dev_s > 0 else 0.0
    result = None
    if rank == 0:
        cpu, sample_gpu, refb = None, None, None
        if world == 1:
            idx = cpu_sample(wl.queries, spec["cpu"])
            sq = [wl.queries[i] for i in idx]
            spk = G.pack_queries(sq)
            G.match_batch(dg, sq, cap=cap, packed=spk, slots=slots, orders=orders, model=model, work_cap=work_cap)
            runs = []
            for _ in range(3):
                G.flush_l2(256 << 20)
                sc, _, _, sinfo = G.match_batch(dg, sq, cap=cap, packed=spk, slots=slots, orders=orders, model=model,
                                                work_cap=work_cap)
                runs.append(sinfo["device_ms"])
            sample_gpu = {"queries": len(sq), "value": len(sq) / (statistics.median(runs) / 1e3),
                          "unit": "queries/s", "device_ms_median_of_3": statistics.median(runs)}
            rate, cores, secs, ccounts = cpu_leg(wl.graph, sq, cap)
            same = bool(np.array_equal(np.asarray(ccounts, np.int64), np.asarray(sc, np.int64)))
            cpu = {"value": rate, "unit": "queries/s", "cores": cores, "kind": "port",
                   "sample": f"the first {len(sq)} queries of the batch with at most {spec['cpu'][0]} vertices "
                             f"(batch indices {idx[0]}..{idx[-1]}), same graph and caps, oracle CPU port of the "
                             f"reference pipeline (plain order) on {cores} threads, {secs:.2f} s; "
                             f"counts equal to the GPU's: {same}",
                   "gpu_same_sample": sample_gpu}
            if args.workload == "rmat22" and not args.no_refbuild:
                refb = reference_build_leg()
        traffic = None
        tf = os.path.join(ROOT, "profiles", "join_traffic.json")
        if os.path.exists(tf) and tot["join_steps"]:
            ratio = json.load(open(tf)).get("traffic_over_alg")
            if ratio:
                traffic = ratio * tot["alg_bytes_join"] / tot["join_steps"]
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
            "data": "synthetic (seeded generators; no public dataset is named for this path)",
            "config": config_of(args, spec, bounds[0][1] - bounds[0][0], world),
            "order": args.order,
            "slots": slots,
            "plain_order": plain,
            "embeddings_per_s": total_rows / dev_s,
            "aborted_at_work_cap": aborted,
            "p50_ms": float(np.percentile(qms_all, 50)) if qms_all else None,
            "p99_ms": float(np.percentile(qms_all, 99)) if qms_all else None,
            "step_ms": [round(x, 1) for x in step_ms],
            # summed per-query device time over slots x step time: how full the
            # slots were (a slice whose last query runs alone lowers it)
            "slot_fill": float(sum(qms_all) / (slots * sum(step_ms))) if step_ms else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "kernel": "join step (k_locate + k_extend_check + k_scan_u32 + k_extend_write)",
                         "peak_source": peak_kind,
                         "achieved_basis": "algorithmic join bytes of the timed steps / the steps' device time "
                                           "(whole step, filter included: a lower bound on the join kernels' rate)",
                         "traffic_per": "join step, DRAM bytes scaled from profiles/join_traffic.json",
                         "alg_bytes_per_step": tot["alg_bytes_join"] / args.steps,
                         "join_steps": tot["join_steps"]},
            "cpu_baseline": cpu,
            "reference_build": refb,
            "e2e": ({"value": None, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 0,
                     "error": e2e_err or "failed on another rank"} if e2e_failed else
                    {"value": e2e_q / e2e_wall, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                     "d2h_bytes_per_step": int(e2e_d2h / max(world, 1)), "rows_per_s": e2e_rows / e2e_wall,
                     "d2h_gb_per_s": e2e_d2h / 1e9 / e2e_wall,
                     "basis": "request server, slice 0 submitted at once (host query arrays in, every embedding "
                              "row to host memory, largest request first, results taken as they finish), after "
                              "one untimed pass", "server_slots": e2e_slots,
                     "host_pool": {"blocks": pool1["blocks"], "pinned_gb": pool1["pinned_bytes"] / 1e9,
                                   "grown_in_timed_pass": pool1["grown"] - pool0["grown"],
                                   "grow_ms_in_timed_pass": pool1["grow_ms"] - pool0["grow_ms"]}}),
            "gpu_launches": int(sum_over_ranks(pg, tot["launches"])),
            "clocks": clk,
            "wall_s": wall,
        }
        print(json.dumps(result), flush=True)
    dg.free()
    if pg is not None:
        pg.destroy_process_group()
    return result


def run_reference(args):
    """The CPU port of the reference pipeline on the fixed sample, each step
    one pass over it; the workload is drawn without loading libgpsm.so."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return None
    import oracle
    from gpsm_b200 import workloads as W
    spec = WORKLOADS[args.workload]
    wl = W.workload(args.workload, source=oracle.GEN_SOURCE)
    idx = cpu_sample(wl.queries, spec["cpu"])
    sq = [wl.queries[i] for i in idx]
    cap = args.cap if args.cap is not None else spec["cap"]
    for _ in range(args.warmup):
        cpu_leg(wl.graph, sq, cap)
    rates, secs_all = [], []
    for _ in range(args.steps):
        rate, cores, secs, _ = cpu_leg(wl.graph, sq, cap)
        rates.append(rate)
        secs_all.append(secs)
    value = len(sq) * args.steps / sum(secs_all)
    nq = len(wl.queries)
    bounds = slice_bounds(nq, spec["slices"])
    result = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(secs_all) / max(args.steps, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded generators; no public dataset is named for this path)",
        "config": config_of(args, spec, bounds[0][1] - bounds[0][0], world),
        "order": "plain (reference heuristic)",
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores, "kind": "port",
                         "sample": f"each step: the first {len(sq)} queries of the batch with at most "
                                   f"{spec['cpu'][0]} vertices (batch indices {idx[0]}..{idx[-1]}), oracle CPU "
                                   f"port of the reference pipeline on {cores} threads; the reference itself has "
                                   f"no CPU implementation of the path"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(result), flush=True)
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat22", choices=sorted(WORKLOADS))
    ap.add_argument("--order", default="learned", choices=["plain", "learned"])
    ap.add_argument("--slots", type=int, default=0, help="engine slots (0 = the tuned count)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-order comparison")
    ap.add_argument("--no-refbuild", action="store_true", help="skip the reference-build leg")
    ap.add_argument("--cap", type=int, default=None, help="embedding cap per query (default: the workload's)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
