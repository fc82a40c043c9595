"""The MLP oracle itself: bfloat16 rounding and gradients by finite differences."""
import numpy as np

from oracle import mlp_oracle as M


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e38], np.float32)
    r = M.to_bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # exactly halfway between 1 and 1+2^-7: ties to even (1.0)
    assert r[2] == 1.0078125      # above halfway: rounds up
    assert r[3] == -2.5


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = (rng.standard_normal(M.P) * 0.2).astype(np.float32)
    p = M.to_bf16(p)  # exact bf16 values so that small perturbations of biases are the only rounding
    x = rng.standard_normal((40, M.F))
    y = rng.standard_normal(40)
    loss, g = M.loss_and_grad(p, x, y)
    # biases are fp32 in the model: check their gradients by central differences
    for i in list(range(M.B1, M.B1 + 5)) + list(range(M.B2, M.B2 + 5)) + [M.B3]:
        e = 1e-3
        pp, pm = p.astype(np.float64).copy(), p.astype(np.float64).copy()
        pp[i] += e
        pm[i] -= e
        lp, _ = M.loss_and_grad(pp.astype(np.float32), x, y)
        lm, _ = M.loss_and_grad(pm.astype(np.float32), x, y)
        assert abs((lp - lm) / (2 * e) - g[i]) < 1e-3 * max(1.0, abs(g[i]))
