"""Test infrastructure, not product code: a float64 numpy restatement of the
separating-axis MLP (24 -> 64 -> 64 -> 16, ReLU, softmax cross-entropy, Adam)
that the CUDA training kernels implement.  It has no counterpart in the
reference engine (the learned proposal is new); it is the checker for the
GPU forward/backward/Adam kernels (gradient check) and nothing else.

Weights are kept as float32 masters and used in the forward pass after
rounding to bfloat16 (round to nearest even), exactly as the kernels do.
"""
import numpy as np

IN, H, OUT = 24, 64, 16
SHAPES = {"w1": (IN, H), "b1": (H,), "w2": (H, H), "b2": (H,), "w3": (H, OUT), "b3": (OUT,)}
ORDER = ("w1", "b1", "w2", "b2", "w3", "b3")


def bf16_round(a):
    """float32 -> bfloat16 (round to nearest even) -> float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounding = 0x7FFF + ((u >> 16) & 1)
    r = ((u + rounding) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    out[nan] = a[nan]
    return out


def forward(params, x):
    """Returns (h1, h2, logits) in float64; weight matrices are bf16-rounded."""
    w1, w2, w3 = (bf16_round(params[k]).astype(np.float64) for k in ("w1", "w2", "w3"))
    b1, b2, b3 = (params[k].astype(np.float64) for k in ("b1", "b2", "b3"))
    x = x.astype(np.float64)
    h1 = np.maximum(x @ w1 + b1, 0.0)
    h2 = np.maximum(h1 @ w2 + b2, 0.0)
    z = h2 @ w3 + b3
    return h1, h2, z


def loss_and_grads(params, x, y):
    """Mean softmax cross-entropy and its gradients w.r.t. every parameter
    (the bf16 rounding of the weights is treated as identity in the backward
    pass, the usual straight-through rule)."""
    h1, h2, z = forward(params, x)
    n = x.shape[0]
    zmax = z.max(axis=1, keepdims=True)
    e = np.exp(z - zmax)
    p = e / e.sum(axis=1, keepdims=True)
    loss = float(np.mean(-np.log(p[np.arange(n), y])))
    dz = p.copy()
    dz[np.arange(n), y] -= 1.0
    dz /= n
    w2 = bf16_round(params["w2"]).astype(np.float64)
    w3 = bf16_round(params["w3"]).astype(np.float64)
    g = {}
    g["w3"] = h2.T @ dz
    g["b3"] = dz.sum(axis=0)
    dh2 = (dz @ w3.T) * (h2 > 0)
    g["w2"] = h1.T @ dh2
    g["b2"] = dh2.sum(axis=0)
    dh1 = (dh2 @ w2.T) * (h1 > 0)
    g["w1"] = x.astype(np.float64).T @ dh1
    g["b1"] = dh1.sum(axis=0)
    return loss, g


def adam(params, grads, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (bias-corrected), float64 state."""
    out = {}
    for k in ORDER:
        m[k] = b1 * m[k] + (1 - b1) * grads[k]
        v[k] = b2 * v[k] + (1 - b2) * grads[k] ** 2
        mh = m[k] / (1 - b1 ** t)
        vh = v[k] / (1 - b2 ** t)
        out[k] = params[k] - lr * mh / (np.sqrt(vh) + eps)
    return out


def init_params(seed=0):
    """He-uniform initialisation (float32), the same recipe as the library's."""
    rng = np.random.default_rng(seed)
    p = {}
    for k in ORDER:
        shp = SHAPES[k]
        if len(shp) == 2:
            lim = np.sqrt(6.0 / shp[0])
            p[k] = rng.uniform(-lim, lim, shp).astype(np.float32)
        else:
            p[k] = np.zeros(shp, np.float32)
    return p
