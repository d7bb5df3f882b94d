"""Contact-manifold reduction on the GPU (rp3dg_reduce_contacts_device and
rp3dg_narrowphase_manifolds_host, through the C ABI) against the reference's
reduced manifolds (committed fixture) and the C oracle: bit-exact kept points,
counts and kept-slot tables."""
import numpy as np
import pytest
import torch

import edgecases
import goldenio
import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes
from test_manifold import assert_reduced_equal

pytestmark = pytest.mark.gpu
GOLDEN = reflib.ROOT + "/tests/golden/"


def _register_hulls(e):
    v, f = edgecases.load_hull()
    m = e.create_convex_mesh(v, f)
    assert e.create_convex_mesh_shape(m) == 0
    assert e.create_convex_mesh_shape(m, edgecases.HULL_SCALE) == 1


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    _register_hulls(c)
    yield c
    c.close()


@pytest.fixture(scope="module")
def port_hulls(port):
    port.lib.rp3do_reset()
    _register_hulls(port)
    return port


def _upload(raw):
    d = engine.DeviceContacts(raw.n, raw.max_contacts)
    for f in goldenio.MANIFOLD_FIELDS:
        getattr(d, f).copy_(torch.from_numpy(np.ascontiguousarray(getattr(raw, f))))
    return d


def _reduce_on_gpu(ctx, pairs, raw):
    dp, dc = engine.DevicePairs(pairs), _upload(raw)
    kept = torch.full((pairs.n, 4), 7, dtype=torch.uint8, device="cuda")
    ctx.reduce_contacts_device(dp, dc, kept)
    ctx.synchronize()
    return dc.to_host(), kept.cpu().numpy()


def test_gpu_reduction_matches_reference_fixture(ctx):
    z = np.load(GOLDEN + "np_manifold.npz")
    for name in goldenio.manifold_groups(z):
        pairs, raw, red, kept = goldenio.unpack_manifold(z, name)
        got, k = _reduce_on_gpu(ctx, pairs, raw)
        assert_reduced_equal(got, red, k, kept, name)


@pytest.mark.parametrize("seed", [211, 212])
def test_gpu_manifolds_match_oracle(ctx, port_hulls, seed):
    """Narrow phase + reduction in one host call against the oracle's narrow
    phase followed by the oracle's reduction."""
    sc = scenes.narrowphase_scene(total_pairs=7 * 4096, seed=seed, hull=edgecases.load_hull())
    ctx.set_shapes(sc.shapes)
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        pg, pp = pairs.slice(0, pairs.n), pairs.slice(0, pairs.n)
        exp, _ = port_hulls.narrowphase(algo, sc.shapes, pp)
        kexp = reflib.reduce_contacts(port_hulls.lib, "rp3do_reduce_contacts", pp, exp)
        got, kgot = ctx.narrowphase_manifolds_host(algo, pg)
        assert_reduced_equal(got, exp, kgot, kexp, name)
        a = np.ascontiguousarray(pg.cache).view(np.uint8)
        b = np.ascontiguousarray(pp.cache).view(np.uint8)
        assert np.array_equal(a, b), (name, "cache")


def test_gpu_reduction_full_size(ctx, port_hulls):
    """The full 1,048,576-pair workload: device narrow phase, then the device
    reduction against the oracle's reduction of the same raw points; reducing
    a reduced manifold again changes nothing (idempotence)."""
    sc = scenes.narrowphase_scene(seed=1234, hull=edgecases.load_hull())
    ctx.set_shapes(sc.shapes)
    for name, (algo, pairs) in sc.batches.items():
        dp = engine.DevicePairs(pairs)
        dc = engine.DeviceContacts(pairs.n)
        ctx.narrowphase_device(algo, dp, dc)
        ctx.synchronize()
        raw = dc.to_host()
        kept = torch.empty((pairs.n, 4), dtype=torch.uint8, device="cuda")
        ctx.reduce_contacts_device(dp, dc, kept)
        ctx.synchronize()
        got, kgot = dc.to_host(), kept.cpu().numpy()
        exp = reflib.copy_contacts(raw)
        kexp = reflib.reduce_contacts(port_hulls.lib, "rp3do_reduce_contacts", pairs, exp)
        assert_reduced_equal(got, exp, kgot, kexp, name)
        assert got.nb_contacts.max() <= 4
        ctx.reduce_contacts_device(dp, dc, kept)
        ctx.synchronize()
        again = dc.to_host()
        assert_reduced_equal(again, got, what=name + " idempotent")
        assert np.array_equal(kept.cpu().numpy()[:, :], np.where(kgot == 255, 255,
                                                                  np.arange(4, dtype=np.uint8)[None, :]))


def test_reduction_empty_and_errors(ctx):
    z = np.zeros(0, np.int32)
    empty = A.HostPairs(z, z, np.zeros((0, 4)), np.zeros((0, 4)), np.zeros((0, 4)), np.zeros((0, 4)))
    out, kept = ctx.narrowphase_manifolds_host(A.ALGO_SPHERE_VS_SPHERE, empty, A.HostContacts(0))
    assert kept.shape == (0, 4)
    pairs, raw, _, _ = goldenio.unpack_manifold(np.load(GOLDEN + "np_manifold.npz"), "box_box")
    dp, dc = engine.DevicePairs(pairs), _upload(raw)
    dc.max_contacts = 0
    with pytest.raises(engine.Rp3dgError):
        ctx.reduce_contacts_device(dp, dc)
    dc.max_contacts = 17
    with pytest.raises(engine.Rp3dgError):
        ctx.reduce_contacts_device(dp, dc)


def test_misaligned_device_arrays_rejected(ctx):
    """A float4 array that is not 16-byte aligned is refused on the host before
    any launch (the kernels read it with 16-byte vector loads)."""
    pairs, raw, _, _ = goldenio.unpack_manifold(np.load(GOLDEN + "np_manifold.npz"), "box_box")
    dp, dc = engine.DevicePairs(pairs), _upload(raw)
    s = dc.struct()
    s.normal_depth = dc.normal_depth.data_ptr() + 4
    pb = dp.struct()
    import ctypes as C
    rc = ctx.lib.rp3dg_reduce_contacts_device(ctx.h, C.byref(pb), C.byref(s), None)
    assert rc == -1 and b"misaligned" in ctx.lib.rp3dg_last_error(ctx.h)
    s = dc.struct()
    rc = ctx.lib.rp3dg_reduce_contacts_device(ctx.h, C.byref(pb), C.byref(s),
                                               torch.empty(4 * pairs.n + 4, dtype=torch.uint8,
                                                           device="cuda").data_ptr() + 1)
    assert rc == -1
    ctx.synchronize()
