"""The float64 MLP oracle (oracle/axis_mlp_oracle.py) pinned by central finite
differences: it has no counterpart in the reference engine, so its analytic
gradients are checked against its own loss."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import axis_mlp_oracle as M  # noqa: E402


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.0078125, -2.5, 3.0e-3, 65504.0], np.float32)
    r = M.bf16_round(x)
    assert r[0] == 1.0 and r[3] == -2.5
    # 1 + 2^-8 is halfway between bf16 neighbours 1 and 1 + 2^-7: ties to even -> 1
    assert r[1] == 1.0
    assert r[2] == np.float32(1.0078125)
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = M.init_params(3)
    # keep weights on the bf16 grid so the loss is smooth in them
    for k in ("w1", "w2", "w3"):
        p[k] = M.bf16_round(p[k])
    for k in ("b1", "b2", "b3"):
        p[k] = rng.normal(0, 0.1, p[k].shape).astype(np.float32)
    x = rng.normal(size=(16, M.IN)).astype(np.float32)
    y = rng.integers(0, M.OUT, 16)
    _, g = M.loss_and_grads(p, x, y)
    # biases are not rounded, so central differences apply directly
    for k in ("b1", "b2", "b3"):
        for idx in [0, 3, p[k].size - 1]:
            h = 1e-6
            pp = {q: v.copy() for q, v in p.items()}
            pm = {q: v.copy() for q, v in p.items()}
            pp[k] = pp[k].astype(np.float64); pm[k] = pm[k].astype(np.float64)
            pp[k].flat[idx] += h
            pm[k].flat[idx] -= h
            num = (M.loss_and_grads(pp, x, y)[0] - M.loss_and_grads(pm, x, y)[0]) / (2 * h)
            assert abs(num - g[k].flat[idx]) < 1e-7 + 1e-4 * abs(num), (k, idx, num, g[k].flat[idx])


def test_oracle_adam_moves_against_gradient():
    p = M.init_params(1)
    g = {k: np.ones_like(v, dtype=np.float64) for k, v in p.items()}
    m = {k: np.zeros_like(v, dtype=np.float64) for k, v in p.items()}
    v = {k: np.zeros_like(v, dtype=np.float64) for k, v in p.items()}
    q = M.adam(p, g, m, v, 1, lr=1e-2)
    for k in M.ORDER:
        assert np.allclose(q[k] - p[k], -1e-2, atol=1e-6)
