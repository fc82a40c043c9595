"""Autotuner for the engine's launch choices.

    python -m gpsm_b200.autotune [--workload rmat22] [--slices 0,7] [--out gpsm_b200/data/tuning.json]

Times whole slices of the benchmark batch (1/20 of the 4,096 queries each,
the bench's own steps, with its cap and work cap) in the learned join order
on the tuned number of slots (device time of the batch, best of two runs
after a warm-up) under every combination of:
  heavy_degree       candidates above it get a block each (filter kernels)
  ext_blocks_per_sm  persistent join-check blocks per SM (at most what the
                     SM holds for the kernel's register count)
  ext_items          candidates per thread of the join-check kernel (4 or 8:
                     its tile is 256 x ext_items candidates; a thread keeps
                     one row's state and list positions across its items)
  filter_team        lanes per candidate in the refinement steps (4, 8 or 32)
  explore_team       lanes per candidate in the exploration steps (8 or 32)
  step_cands         candidates one join step may admit
  slots              engine slots running queries at once
and writes the fastest combination to --out; gpsm_b200.init() applies it.
Whole slices keep the queries that run to the work cap: they decide the
step budget (a budget whose scratch outgrows L2 slows every long query) and
a sample of quick queries alone picked the wrong one. --queries N instead
times N quick queries (device time under --max-ms each).
The grid keeps what earlier sweeps left open (a 4,096 hub threshold, 6
check blocks per SM, 4 candidates per check thread and the 2^23 step budget
won every sweep; 32-lane refinement teams lost each time).
Slot counts are compared one process each (--slots; a process sizes every
slot pool from the memory left free when the pool is created, so a second
pool in the same process would get less): the grid keeps one count.
"""
import argparse
import itertools
import json
import os
import time

import numpy as np

from . import DeviceGraph, get_tuning, init, match, match_batch, set_tuning
from . import learned as L
from . import workloads as W

GRID = dict(heavy_degree=[4096], ext_blocks_per_sm=[6], ext_items=[4], filter_team=[4, 8],
            explore_team=[8, 32], step_cands=[1 << 23], slots=[12])
NSLICES = 20  # the bench's slices of the batch


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="rmat22")
    ap.add_argument("--work-cap", type=int, default=5_000_000_000)
    ap.add_argument("--slices", default="0,7", help="bench slices to time (of 20)")
    ap.add_argument("--queries", type=int, default=0, help="time this many quick queries instead")
    ap.add_argument("--cap", type=int, default=10_000_000)
    ap.add_argument("--max-ms", type=float, default=200.0)
    ap.add_argument("--slots", type=int, default=0, help="the slot count to tune at (0 = the grid's)")
    ap.add_argument("--grid", default="", help='JSON object replacing grid entries, e.g. {"step_cands": [8388608]}')
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                                  "tuning.json"))
    args = ap.parse_args()
    init(0, tuning_file=None)
    default = get_tuning()
    wl = W.workload(args.workload, count=max(args.queries * 3, 100) if args.queries else None)
    dg = DeviceGraph(wl.graph)
    model = L.load(0)
    sample = []
    if args.queries:
        for q in wl.queries:
            out = match(dg, q, cap=args.cap, count_only=True, order="learned", model=model,
                        work_cap=2_000_000_000)
            if out.info["device_ms"] < args.max_ms:
                sample.append(q)
            if len(sample) >= args.queries:
                break
    else:
        nq = len(wl.queries)
        for sl in (int(x) for x in args.slices.split(",")):
            sample.extend(wl.queries[nq * sl // NSLICES: nq * (sl + 1) // NSLICES])
    if args.grid:
        for k, v in json.loads(args.grid).items():
            if k not in GRID:
                raise SystemExit(f"unknown grid entry {k}")
            GRID[k] = list(v)
    if args.slots:
        GRID["slots"] = [args.slots]
    results = []
    keys = list(GRID)
    for combo in itertools.product(*[GRID[k] for k in keys]):
        choice = dict(zip(keys, combo))
        set_tuning(**choice)
        def run():
            return match_batch(dg, sample, cap=args.cap, slots=choice["slots"], orders="learned", model=model,
                               work_cap=args.work_cap)

        run()  # warm-up
        best = min(run()[3]["device_ms"] for _ in range(2))
        results.append(dict(choice=choice, device_ms=best))
        print(json.dumps(results[-1]), flush=True)
    set_tuning(**default)
    best = min(results, key=lambda r: r["device_ms"])
    base = [r for r in results if all(r["choice"][k] == default.get(k, r["choice"][k]) for k in keys)]
    out = dict(choice=best["choice"], device_ms=best["device_ms"],
               default_ms=base[0]["device_ms"] if base else None, workload=args.workload,
               sample_queries=len(sample), slices=None if args.queries else args.slices, cap=args.cap, when=time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
               all=results)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    print("best", json.dumps(best), "default", out["default_ms"], flush=True)


if __name__ == "__main__":
    main()
