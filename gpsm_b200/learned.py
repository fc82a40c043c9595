"""Learned join order: training-sample collection, training and evaluation.

A sample is one join step of one query under one vertex order: the step's
16 features (gpsm_order_features, computed from the filter statistics) and
its measured log2 expansion log2((rows_out + 1) / (rows_in + 1)), where
rows_in are the rows of the current width the engine extended and rows_out
the rows it produced (both from gpsm_last_levels). Every query contributes
the plain order and a few random connected orders, so the model sees good
and bad steps. Runs are capped (embedding cap and work cap) to keep the
collection bounded; the last level of a capped run is left out because the
cap truncates its output.
"""
import os

import numpy as np

from . import DeviceGraph, Model, debug_filter, last_levels, match, order_features  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "order_model.npz")


def random_order(q, rng):
    adj = [set() for _ in range(q.n)]
    for a, b in np.asarray(q.edges).tolist():
        adj[a].add(b)
        adj[b].add(a)
    order = [int(rng.integers(q.n))]
    seen = set(order)
    while len(order) < q.n:
        cand = sorted({w for u in order for w in adj[u]} - seen)
        v = cand[int(rng.integers(len(cand)))]
        order.append(v)
        seen.add(v)
    return order


def step_samples(dg, q, filt, order, cap, work_cap):
    """Run one order and return (features, targets, run info)."""
    out = match(dg, q, cap=cap, order=order, count_only=True, work_cap=work_cap)
    lin, lc, lout = last_levels(q.n)
    feats = order_features(dg, q, filt, out.pos2id)
    xs, ys = [], []
    truncated = out.capped or out.info["aborted"]
    last_w = max([w for w in range(1, q.n) if lin[w] > 0], default=0)
    for k in range(1, q.n):  # step k extends width k to width k+1
        if lin[k] == 0:
            continue
        if truncated and k == last_w:
            continue
        xs.append(feats[k - 1])
        ys.append(np.log2((float(lout[k + 1]) + 1.0) / (float(lin[k]) + 1.0)))
    return xs, ys, out


def collect(dg, queries, orders_per_query=2, cap=100_000, work_cap=200_000_000, seed=0, log=None):
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for i, q in enumerate(queries):
        if q.n < 3:
            continue
        filt = debug_filter(dg, q)
        if filt["empty"]:
            continue
        orders = [None] + [random_order(q, rng) for _ in range(orders_per_query - 1)]
        for o in orders:
            xs, ys, _ = step_samples(dg, q, filt, o, cap, work_cap)
            X.extend(xs)
            Y.extend(ys)
        if log and (i + 1) % 500 == 0:
            log(f"collected {i + 1} queries, {len(Y)} samples")
    return np.asarray(X, np.float32).reshape(-1, 16), np.asarray(Y, np.float32)


def train(X, Y, device=0, seed=0, epochs=40, batch=2048, lr=2e-3):
    m = Model(device, seed)
    loss = m.train(X, Y, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return m, loss


def save(model, path=WEIGHTS, **meta):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=model.get(), **{k: np.asarray(v) for k, v in meta.items()})


def load(device=0, path=WEIGHTS):
    z = np.load(path)
    return Model(device, params=z["params"])


def order_stats(dg, q, order, cap, model=None, work_cap=0):
    """Embeddings, join time and table sizes of one query under one order."""
    out = match(dg, q, cap=cap, order=order, model=model, count_only=True, work_cap=work_cap)
    lin, lc, lout = last_levels(q.n)
    return dict(count=out.count, capped=out.capped, aborted=bool(out.info["aborted"]), join_ms=out.info["join_ms"],
                device_ms=out.info["device_ms"],
                rows=int(lin[1:].sum()), cands=int(out.info["cands_scanned"]), peak=int(lout[2:].max()) if q.n > 1 else 0,
                pos2id=[int(x) for x in out.pos2id], fallback=int(out.info["order_fallback"]),
                predicted_work=float(out.info["predicted_work"]),
                predicted_work_plain=float(out.info["predicted_work_plain"]),
                attempts=int(out.info["order_attempts"]))
