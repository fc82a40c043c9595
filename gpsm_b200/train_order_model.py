"""Train the learned join-order model on the GPU and evaluate it.

    python -m gpsm_b200.train_order_model [--train 5000] [--eval 200] [--regret 20] [--out DIR]

1. Samples: the rmat20 graph (R-MAT 2^20, 16 Mi edges, Zipf labels) and 5,000
   separately seeded training queries of 4..32 vertices (half tree, half
   dense); each query runs under the plain order and a random connected
   order, and every join step becomes one (features, log2 expansion) sample.
2. Training: Adam on the GPU (gpsm_model_train), BF16 weights, FP32 masters.
3. Evaluation on held-out queries of the same shape (the rmat20_mix set):
   learned vs plain order, embeddings per query (identical when neither run
   is capped), join time and table sizes.
4. Regret on small queries (<= 6 vertices): every connected order is run;
   the best one is compared with the learned and the plain order.
Writes order_model.npz (weights) and order_eval.json to --out.
"""
import argparse
import itertools
import json
import os
import time

import numpy as np

from . import DeviceGraph, init
from . import learned as L
from . import workloads as W


def connected_orders(q):
    adj = [set() for _ in range(q.n)]
    for a, b in np.asarray(q.edges).tolist():
        adj[a].add(b)
        adj[b].add(a)
    for perm in itertools.permutations(range(q.n)):
        ok = True
        seen = {perm[0]}
        for v in perm[1:]:
            if not (adj[v] & seen):
                ok = False
                break
            seen.add(v)
        if ok:
            yield list(perm)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=5000)
    ap.add_argument("--eval", type=int, default=200)
    ap.add_argument("--regret", type=int, default=20)
    ap.add_argument("--cap", type=int, default=10_000_000)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "data"))
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--eval-only", action="store_true", help="load the committed weights, skip training")
    ap.add_argument("--work-cap", type=int, default=2_000_000_000,
                    help="candidates a join may scan in the evaluation (bounds plain-order blowups)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    init(0)
    t0 = time.time()
    g = W.graph_for("rmat20")
    dg = DeviceGraph(g)
    if args.eval_only:
        model = L.load(0)
        z = np.load(L.WEIGHTS)
        loss, val_mse, base_mse, nsamples = None, float(z["val_mse"]), float(z["base_mse"]), int(z["samples"])
    else:
        train_q = W.workload("rmat20_train", count=args.train).queries
        X, Y = L.collect(dg, train_q, orders_per_query=2, log=print)
        nsamples = len(Y)
        print(f"samples {len(Y)} from {len(train_q)} queries in {time.time() - t0:.1f}s", flush=True)
        rng = np.random.default_rng(1)
        idx = rng.permutation(len(Y))
        nval = max(1, len(Y) // 10)
        val, tr = idx[:nval], idx[nval:]
        model, loss = L.train(X[tr], Y[tr], epochs=args.epochs)
        pred = model.predict(X[val])
        val_mse = float(np.mean((pred - Y[val]) ** 2))
        base_mse = float(np.mean((Y[val] - Y[tr].mean()) ** 2))
        print(f"train loss {loss:.4f} val mse {val_mse:.4f} (constant predictor {base_mse:.4f})", flush=True)
        L.save(model, os.path.join(args.out, "order_model.npz"), train_queries=args.train, samples=len(Y),
               val_mse=val_mse, base_mse=base_mse)
    # evaluation on held-out queries
    ev = W.workload("rmat20_mix", count=args.eval).queries
    res = []
    for i, q in enumerate(ev):
        p = L.order_stats(dg, q, None, args.cap, work_cap=args.work_cap)
        l = L.order_stats(dg, q, "learned", args.cap, model=model, work_cap=args.work_cap)
        res.append(dict(i=i, n=q.n, m=q.m, plain=p, learned=l))
        if (i + 1) % 25 == 0:
            print(f"eval {i + 1} plain_ms {sum(r['plain']['device_ms'] for r in res):.0f} "
                  f"learned_ms {sum(r['learned']['device_ms'] for r in res):.0f}", flush=True)
    same = all((r["plain"]["count"] == r["learned"]["count"]) or r["plain"]["capped"] or r["learned"]["capped"]
               or r["plain"].get("aborted") or r["learned"].get("aborted") for r in res)
    tot = {k: {m: float(sum(r[k][m] for r in res)) for m in ("join_ms", "device_ms", "rows", "cands")}
           for k in ("plain", "learned")}
    print(json.dumps(dict(eval_queries=len(res), counts_agree=same, totals=tot)), flush=True)
    # regret on small queries
    small = [q for q in W.workload("rmat20_mix", count=1000).queries if q.n <= 6][: args.regret]
    print(f"regret on {len(small)} small queries", flush=True)
    reg = []
    for q in small:
        runs = [(o, L.order_stats(dg, q, o, 1_000_000)) for o in connected_orders(q)]
        best_t = min(r["join_ms"] for _, r in runs)
        best_rows = min(r["rows"] for _, r in runs)
        p = L.order_stats(dg, q, None, 1_000_000)
        l = L.order_stats(dg, q, "learned", 1_000_000, model=model)
        reg.append(dict(n=q.n, orders=len(runs), best_ms=best_t, best_rows=best_rows, plain_ms=p["join_ms"],
                        plain_rows=p["rows"], learned_ms=l["join_ms"], learned_rows=l["rows"],
                        plain_peak=p["peak"], learned_peak=l["peak"], best_peak=min(r["peak"] for _, r in runs)))
    out = dict(samples=nsamples, val_mse=val_mse, base_mse=base_mse, train_loss=loss, eval=res, totals=tot,
               counts_agree=same, regret=reg, seconds=time.time() - t0)
    with open(os.path.join(args.out, "order_eval.json"), "w") as f:
        json.dump(out, f)
    print("regret", json.dumps(reg[:5]), flush=True)
    print(f"done in {time.time() - t0:.1f}s", flush=True)


if __name__ == "__main__":
    main()
