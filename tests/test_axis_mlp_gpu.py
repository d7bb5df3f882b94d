"""Learned separating-axis proposal on the GPU: the hand-written training
kernels against the float64 oracle (gradients, Adam), tensor-core inference
against the oracle's arg-max, training on labels from the engine's own SAT,
and the narrow phase with proposals on: contacts bit-identical to plain SAT."""
import os
import sys

import numpy as np
import pytest

import edgecases
import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes

sys.path.insert(0, os.path.join(reflib.ROOT, "oracle"))
import axis_mlp_oracle as M  # noqa: E402

pytestmark = pytest.mark.gpu


def _split(p):
    out, k = {}, 0
    for name in M.ORDER:
        size = int(np.prod(M.SHAPES[name]))
        out[name] = p[k:k + size].reshape(M.SHAPES[name]).astype(np.float32)
        k += size
    return out


def _flat(d):
    return np.concatenate([np.asarray(d[k], np.float64).ravel() for k in M.ORDER])


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    v, f = edgecases.load_hull()
    c.create_convex_mesh_shape(c.create_convex_mesh(v, f))
    yield c
    c.close()


def test_gradients_match_oracle(ctx):
    import torch
    mlp = engine.AxisMLP(ctx, seed=11)
    p = mlp.params()
    rng = np.random.default_rng(1)
    n = 3000
    x = rng.normal(size=(n, M.IN)).astype(np.float32)
    y = rng.integers(0, M.OUT, n).astype(np.uint8)
    g, loss = mlp.grads(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda())
    g = g.cpu().numpy().astype(np.float64)
    ref_loss, ref = M.loss_and_grads(_split(p), x, y.astype(np.int64))
    assert abs(loss - ref_loss) < 1e-4 * max(1.0, abs(ref_loss))
    gd = _split(g.astype(np.float32))
    for k in M.ORDER:
        err = np.linalg.norm(gd[k].astype(np.float64) - ref[k]) / max(np.linalg.norm(ref[k]), 1e-12)
        assert err < 2e-3, (k, err)


def test_adam_step_matches_oracle(ctx):
    import torch
    mlp = engine.AxisMLP(ctx, seed=5)
    p0 = _split(mlp.params())
    rng = np.random.default_rng(2)
    x = rng.normal(size=(2048, M.IN)).astype(np.float32)
    y = rng.integers(0, M.OUT, 2048).astype(np.uint8)
    _, g = M.loss_and_grads(p0, x, y.astype(np.int64))
    mlp.train_step(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), lr=1e-3)
    p1 = _split(mlp.params())
    zeros = {k: np.zeros_like(v, dtype=np.float64) for k, v in p0.items()}
    q = M.adam(p0, g, dict(zeros), {k: v.copy() for k, v in zeros.items()}, 1, lr=1e-3)
    for k in M.ORDER:
        # where the gradient is not tiny the first Adam step is -lr * sign(g)
        sig = np.abs(g[k]) > 1e-5
        assert np.allclose(p1[k][sig], q[k][sig], atol=2e-6), k
        assert np.all(np.abs(p1[k] - p0[k]) <= 1e-3 * 1.001), k


def test_tensor_core_predict_matches_oracle_argmax(ctx):
    import torch
    mlp = engine.AxisMLP(ctx, seed=3)
    rng = np.random.default_rng(3)
    # give the output layer some spread so the arg-max is not a coin flip
    p = _split(mlp.params())
    p["b3"] = rng.normal(0, 0.5, p["b3"].shape).astype(np.float32)
    mlp.set_params(_flat(p).astype(np.float32))
    x = rng.normal(size=(4096 + 17, M.IN)).astype(np.float32)
    got = mlp.predict(torch.from_numpy(x).cuda()).cpu().numpy()
    _, _, z = M.forward(p, x)
    exp = z.argmax(axis=1)
    agree = float(np.mean(got == exp))
    # bf16 activations can only flip near-ties
    assert agree > 0.97, agree


@pytest.fixture(scope="module")
def trained(ctx):
    """An MLP trained on box-box and hull-box pairs labelled by the plain SAT."""
    import torch
    sc = scenes.narrowphase_scene(total_pairs=7 * 60000, seed=505, names=("box_box", "hull_box"),
                                  hull=edgecases.load_hull())
    ctx.set_shapes(sc.shapes)
    mlp = engine.AxisMLP(ctx, seed=7)
    xs, ys = [], []
    for name in ("box_box", "hull_box"):
        algo, pairs = sc.batches[name]
        pairs.cache = A.fresh_cache(pairs.n)
        dp = engine.DevicePairs(pairs)
        out = engine.DeviceContacts(pairs.n)
        ctx.narrowphase_device(algo, dp, out)
        xs.append(mlp.features(dp))
        ys.append(mlp.labels(dp, out))
    ctx.synchronize()
    x, y = torch.cat(xs), torch.cat(ys)
    n = x.shape[0]
    perm = torch.randperm(n, generator=torch.Generator().manual_seed(1)).cuda()
    x, y = x[perm].contiguous(), y[perm].contiguous()
    ntr = int(0.8 * n)
    losses = engine.train_axis_mlp(ctx, mlp, x[:ntr], y[:ntr], epochs=6, batch=4096, lr=3e-3)
    return dict(mlp=mlp, x_test=x[ntr:], y_test=y[ntr:], losses=losses, scene=sc)


def test_training_on_sat_labels(trained):
    losses = trained["losses"]
    assert losses[-1] < losses[0] * 0.8, losses
    pred = trained["mlp"].predict(trained["x_test"]).cpu().numpy()
    y = trained["y_test"].cpu().numpy()
    acc = float(np.mean(pred == y))
    majority = float(np.max(np.bincount(y, minlength=16))) / len(y)
    print(f"held-out accuracy {acc:.3f} (majority class {majority:.3f}), losses {losses}")
    assert acc > majority + 0.05, (acc, majority)


def _frames(ctx, sc, names, enable_mlp, mlp):
    """Two frames (fresh caches, then moved poses with the caches) of each batch."""
    rng = np.random.default_rng(9)
    res = {}
    for name in names:
        algo, pairs = sc.batches[name]
        p = pairs.slice(0, pairs.n)
        p.cache = A.fresh_cache(p.n)
        mlp.enable(enable_mlp)
        o1 = ctx.narrowphase_host(algo, p)
        nxt = reflib.perturb_pairs(p, np.random.default_rng(17))
        nxt.cache = reflib.next_frame_cache(p.cache, o1)
        o2 = ctx.narrowphase_host(algo, nxt)
        mlp.enable(False)
        res[name] = (o1, p.cache.copy(), o2, nxt.cache.copy())
    return res


def test_learned_sat_keeps_contacts_bit_identical(ctx, trained):
    mlp = trained["mlp"]
    sc = scenes.narrowphase_scene(total_pairs=7 * 20000, seed=606, names=("box_box", "hull_box"),
                                  hull=edgecases.load_hull())
    ctx.set_shapes(sc.shapes)
    names = ("box_box", "hull_box")
    plain = _frames(ctx, sc, names, False, mlp)
    mlp.stats(clear=True)
    learned = _frames(ctx, sc, names, True, mlp)
    tested, confirmed = mlp.stats(clear=True)
    assert tested > 0 and confirmed > 0, (tested, confirmed)
    for name in names:
        for f in (0, 2):
            a, b = plain[name][f], learned[name][f]
            mism = reflib.compare_contacts(b, a, a.n)
            assert all(v == 0 for v in mism.values()), (name, f, mism)
            ca = plain[name][f + 1].view(np.uint8).reshape(-1, 16)
            cb = learned[name][f + 1].view(np.uint8).reshape(-1, 16)
            diff = np.any(ca != cb, axis=1)
            # caches may differ only where the pair is separated (no contact)
            assert not np.any(diff & (a.is_colliding != 0)), name
    # the frame-2 caches of colliding pairs agree, so the two runs stay in step
    print(f"proposals tested {tested}, confirmed {confirmed}")
