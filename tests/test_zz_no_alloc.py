"""rp3dg_axis_mlp_grads_noalloc, the gradient entry point that allocates no
device memory (for callers whose host application forbids allocations once
the engine runs), called through the C ABI and checked against
rp3dg_axis_mlp_grads on two calls in a row.  This file is collected last so
that a run stopping at the first failure has already run every other test;
it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import edgecases
from reactphysics3d_b200 import engine

pytestmark = pytest.mark.gpu
MAX_SAMPLES = 4096


@pytest.fixture(scope="module")
def setup(cuda_lib):
    import torch
    ctx = engine.Context(0)
    v, f = edgecases.load_hull()
    ctx.create_convex_mesh_shape(ctx.create_convex_mesh(v, f))
    mlp = engine.AxisMLP(ctx, seed=23)
    L = ctx.lib
    L.rp3dg_axis_mlp_grads_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                               C.c_void_p]
    yield ctx, mlp, L, torch
    ctx.close()


def _inputs(torch, n, seed):
    rng = np.random.default_rng(seed)
    x = torch.from_numpy(rng.normal(size=(n, engine.MLP_FEATURES)).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.integers(0, engine.MLP_CLASSES, n).astype(np.uint8)).cuda()
    torch.cuda.synchronize()
    return x, y


def _noalloc(ctx, L, torch, x, y):
    g = torch.empty(engine.MLP_NPARAMS, dtype=torch.float32, device="cuda")
    loss = C.c_float()
    torch.cuda.synchronize()
    rc = L.rp3dg_axis_mlp_grads_noalloc(ctx.h, x.data_ptr(), y.data_ptr(), int(x.shape[0]), g.data_ptr(),
                                        C.addressof(loss))
    assert rc == 0, L.rp3dg_last_error(ctx.h)
    ctx.synchronize()
    return g.cpu().numpy(), loss.value


def test_noalloc_matches_allocating_entry_point_twice(setup):
    ctx, mlp, L, torch = setup
    # two calls in a row with different inputs and sizes: the second must not
    # see anything left in the shared scratch by the first
    for n, seed in ((3000, 1), (1000, 2), (MAX_SAMPLES, 3)):
        x, y = _inputs(torch, n, seed)
        g_ref, loss_ref = mlp.grads(x, y)
        g_ref = g_ref.cpu().numpy()
        g, loss = _noalloc(ctx, L, torch, x, y)
        # same kernels, same summation order: identical gradients; the loss
        # is summed with atomics across blocks, so it may differ in the last bits
        scale = np.maximum(np.abs(g_ref).max(), 1e-12)
        assert np.max(np.abs(g - g_ref)) <= 2e-3 * scale, n
        assert np.array_equal(g, g_ref), n
        assert abs(loss - loss_ref) <= 1e-5 * max(1.0, abs(loss_ref)), (loss, loss_ref)


def test_noalloc_rejects_batches_above_its_limit(setup):
    ctx, mlp, L, torch = setup
    x, y = _inputs(torch, MAX_SAMPLES + 1, 4)
    g = torch.empty(engine.MLP_NPARAMS, dtype=torch.float32, device="cuda")
    rc = L.rp3dg_axis_mlp_grads_noalloc(ctx.h, x.data_ptr(), y.data_ptr(), MAX_SAMPLES + 1, g.data_ptr(), None)
    assert rc == engine.RP3DG_ECAPACITY
    assert b"4096" in L.rp3dg_last_error(ctx.h)
