"""Learned join order on the GPU: gradients against the numpy oracle,
inference, training, exactness of learned orders, the memory-budget
fallback, and what the trained model gains over the plain order."""
import os

import numpy as np
import pytest

import oracle
from oracle import mlp_oracle as MO
from gpsm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _params(seed, scale=0.3):
    rng = np.random.default_rng(seed)
    return MO.to_bf16((rng.standard_normal(MO.P) * scale).astype(np.float32))


def test_gradients_match_oracle(gpu):
    m = gpu.Model(0, seed=1, params=_params(3))
    rng = np.random.default_rng(5)
    x = rng.standard_normal((333, 16)).astype(np.float32)
    y = rng.standard_normal(333).astype(np.float32)
    loss, g = m.grad(x, y)
    ref_loss, ref_g = MO.loss_and_grad(m.get(), x, y)
    assert abs(loss - ref_loss) <= 1e-3 * max(1.0, abs(ref_loss))
    scale = np.abs(ref_g).max()
    # FP32 accumulation on the GPU vs float64 here
    assert np.allclose(g, ref_g, rtol=2e-3, atol=2e-5 * scale)


def test_predict_matches_oracle(gpu):
    m = gpu.Model(0, params=_params(7))
    x = np.random.default_rng(8).standard_normal((1000, 16)).astype(np.float32)
    ref, _ = MO.forward(m.get(), x)
    assert np.allclose(m.predict(x), ref, rtol=1e-4, atol=1e-4)


def test_training_fits_a_smooth_target(gpu):
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, (8192, 16)).astype(np.float32)
    y = (np.maximum(x[:, 0] + x[:, 1], 0) * 3 - x[:, 2] * x[:, 3] + 0.5 * x[:, 4]).astype(np.float32)
    m = gpu.Model(0, seed=2)
    l0 = float(np.mean((m.predict(x) - y) ** 2))
    m.train(x, y, epochs=40, batch=512, lr=3e-3)
    l1 = float(np.mean((m.predict(x) - y) ** 2))
    assert l1 < 0.1 * l0


@pytest.fixture(scope="module")
def small_dg(gpu, small_er):
    return gpu.DeviceGraph(small_er.graph)


def test_learned_order_returns_the_same_embeddings(gpu, small_er, small_dg):
    m = gpu.Model(0, seed=4)  # untrained: the order is arbitrary, the set is not
    for q in small_er.queries:
        base = gpu.match(small_dg, q)
        out = gpu.match(small_dg, q, order="learned", model=m)
        assert sorted(map(tuple, out.embeddings().tolist())) == sorted(map(tuple, base.embeddings().tolist()))
    g = W.rmat_graph(12, 24000, 12, 1.0, seed=5)
    dg = gpu.DeviceGraph(g)
    for k in range(6):
        q = W.random_walk_query(g, 5 + k % 3, 77 + k, W.MODE_DENSE, 0.5)
        rows, cnt = oracle.enumerate_embeddings(g, q, cap=300000)
        if cnt >= 300000:
            continue
        out = gpu.match(dg, q, order="learned", model=m)
        assert sorted(map(tuple, out.embeddings().tolist())) == [tuple(r) for r in rows.tolist()]


def test_memory_budget_falls_back_to_plain_order(gpu, small_er, small_dg):
    m = gpu.Model(0, seed=4)
    q = small_er.queries[0]
    plain = gpu.match(small_dg, q)
    out = gpu.match(small_dg, q, order="learned", model=m, memory_budget=1)
    assert out.info["order_fallback"] == 1
    assert np.array_equal(out.pos2id, plain.pos2id)
    assert np.array_equal(out.rows, plain.rows)


def test_race_restarts_return_the_finishing_orders_rows(gpu):
    """A learned plan takes turns with the plain order under growing work
    shares; whichever order finishes, the rows are exactly those of a match
    in that order (restarts leave nothing behind)."""
    from gpsm_b200 import learned as L
    model = L.load(0) if os.path.exists(L.WEIGHTS) else gpu.Model(0, seed=4)
    g = W.rmat_graph(12, 24000, 12, 1.0, seed=5)
    dg = gpu.DeviceGraph(g)
    old = gpu.get_tuning()
    gpu.set_tuning(race_share=2048)
    raced = 0
    try:
        for k in range(40):
            q = W.random_walk_query(g, 6 + k % 4, 300 + k, W.MODE_DENSE if k % 2 else W.MODE_TREE, 0.5)
            for cap in (200_000, 5000):
                out = gpu.match(dg, q, cap=cap, order="learned", model=model)
                ref = gpu.match(dg, q, cap=cap, order=list(out.pos2id))
                assert out.count == ref.count
                assert np.array_equal(out.embeddings(), ref.embeddings())
                raced += out.info["order_attempts"] >= 2
    finally:
        gpu.set_tuning(race_share=old["race_share"])
    assert raced > 0


def test_trained_model_reduces_join_work(gpu):
    from gpsm_b200 import learned as L
    if not os.path.exists(L.WEIGHTS):
        pytest.skip("no trained weights")
    model = L.load(0)
    wl = W.workload("rmat20_mix", count=40)
    dg = gpu.DeviceGraph(wl.graph)
    plain_rows = learned_rows = 0
    for q in wl.queries:
        p = L.order_stats(dg, q, None, 1_000_000, work_cap=2_000_000_000)
        l = L.order_stats(dg, q, "learned", 1_000_000, model=model, work_cap=2_000_000_000)
        if not p["capped"] and not l["capped"]:
            assert p["count"] == l["count"]
        plain_rows += p["cands"]
        learned_rows += l["cands"]
    # candidates scanned by the joins: a deterministic measure of join work
    assert learned_rows < 0.8 * plain_rows, (learned_rows, plain_rows)
