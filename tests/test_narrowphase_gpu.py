"""CUDA narrow phase (librp3dg.so, called through the C ABI) against the
reference engine's outputs: bit-exact for every field (flags, contact counts,
normals, depths, local points, temporal-coherence caches)."""
import numpy as np
import pytest

import edgecases
import goldenio
import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes

pytestmark = pytest.mark.gpu
GOLDEN = reflib.ROOT + "/tests/golden/"


def _assert_same(got, exp, cache_got=None, cache_exp=None, what=""):
    mism = reflib.compare_contacts(got, exp, exp.n)
    assert all(v == 0 for v in mism.values()), (what, mism)
    if cache_exp is not None:
        a = np.ascontiguousarray(cache_got).view(np.uint8).reshape(-1, 16)
        b = np.ascontiguousarray(cache_exp).view(np.uint8).reshape(-1, 16)
        assert np.array_equal(a, b), (what, "cache", np.argwhere(a != b)[:5])


def _register_hulls(e):
    """The unscaled and the scaled hull instance (ids 0 and 1 in a fresh
    context); returns their ids."""
    v, f = edgecases.load_hull()
    m = e.create_convex_mesh(v, f)
    return e.create_convex_mesh_shape(m), e.create_convex_mesh_shape(m, edgecases.HULL_SCALE)


def _remap_meshes(shapes, ids):
    """The shape table with convex-mesh instance k renamed ids[k] (the
    reference harness keeps its meshes for the whole process, so its ids
    depend on what ran before)."""
    s = np.array(shapes, copy=True)
    conv = s["kind"] == A.SHAPE_CONVEX_MESH
    s["mesh"][conv] = np.asarray(ids)[s["mesh"][conv]]
    return s


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    assert _register_hulls(c) == (0, 1)
    yield c
    c.close()


@pytest.fixture(scope="module")
def port_hulls(port):
    port.lib.rp3do_reset()
    assert _register_hulls(port) == (0, 1)
    return port


@pytest.mark.parametrize("fixture", ["np_scene.npz", "np_edge.npz"])
@pytest.mark.parametrize("api", ["host", "device"])
def test_gpu_matches_golden(ctx, fixture, api):
    z = np.load(GOLDEN + fixture)
    ctx.set_shapes(z["shapes"])
    for pre in goldenio.case_prefixes(z):
        algo, clip, pairs, exp, cache_exp = goldenio.unpack_case(z, pre)
        if api == "host":
            got = ctx.narrowphase_host(algo, pairs, A.HostContacts(pairs.n, exp.max_contacts), clip=clip)
            cache_got = pairs.cache
        else:
            dp = engine.DevicePairs(pairs)
            dout = engine.DeviceContacts(pairs.n, exp.max_contacts)
            ctx.narrowphase_device(algo, dp, dout, clip=clip)
            ctx.synchronize()
            got, cache_got = dout.to_host(), dp.host_cache()
        _assert_same(got, exp, cache_got, cache_exp, pre + api)


def test_gpu_mesh_tables_match_oracle(ctx, port_hulls):
    for inst in (0, 1):
        a, b = ctx.mesh_tables(inst), port_hulls.mesh_tables(inst)
        assert np.array_equal(a["half_edges"], b["half_edges"])
        assert np.array_equal(a["face_edge"], b["face_edge"])
        assert np.array_equal(a["face_normals"].view(np.uint32), b["face_normals"].view(np.uint32))
        assert np.array_equal(a["centroid"].view(np.uint32), b["centroid"].view(np.uint32))


@pytest.mark.parametrize("seed", [101, 102, 103])
def test_gpu_matches_oracle_two_frames(ctx, port_hulls, seed):
    """Fresh caches, then a second frame with moved poses and the first frame's
    caches (temporal coherence), on a seeded scene of all seven batches."""
    sc = scenes.narrowphase_scene(total_pairs=7 * 4096, seed=seed, hull=edgecases.load_hull())
    ctx.set_shapes(sc.shapes)
    rng = np.random.default_rng(seed)
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        pg, pp = pairs.slice(0, pairs.n), pairs.slice(0, pairs.n)
        b, _ = port_hulls.narrowphase(algo, sc.shapes, pp)
        g = ctx.narrowphase_host(algo, pg)
        _assert_same(g, b, pg.cache, pp.cache, name + " frame 1")
        nxt = reflib.perturb_pairs(pp, rng)
        nxt.cache = reflib.next_frame_cache(pp.cache, b)
        pg2, pp2 = nxt.slice(0, nxt.n), nxt.slice(0, nxt.n)
        b2, _ = port_hulls.narrowphase(algo, sc.shapes, pp2)
        g2 = ctx.narrowphase_host(algo, pg2)
        _assert_same(g2, b2, pg2.cache, pp2.cache, name + " frame 2")


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build oracle/_ref not present")
def test_gpu_matches_reference_build(ctx):
    ref = reflib.RefEngine("f32")
    ref_shapes = None
    sc = scenes.narrowphase_scene(total_pairs=7 * 2048, seed=77, hull=edgecases.load_hull())
    ref_shapes = _remap_meshes(sc.shapes, _register_hulls(ref))
    ctx.set_shapes(sc.shapes)
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        pr, pg = pairs.slice(0, pairs.n), pairs.slice(0, pairs.n)
        a, _ = ref.narrowphase(algo, ref_shapes, pr)
        g = ctx.narrowphase_host(algo, pg)
        _assert_same(g, a, pg.cache, pr.cache, name)


def test_empty_batch_and_errors(ctx):
    z = np.load(GOLDEN + "np_edge.npz")
    ctx.set_shapes(z["shapes"])
    empty = A.HostPairs(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, 4)), np.zeros((0, 4)),
                        np.zeros((0, 4)), np.zeros((0, 4)))
    ctx.narrowphase_host(A.ALGO_SPHERE_VS_SPHERE, empty, A.HostContacts(0))
    algo, clip, pairs, exp, _ = goldenio.unpack_case(z, "sphere_sphere_")
    with pytest.raises(engine.Rp3dgError):
        ctx.narrowphase_host(7, pairs)
    with pytest.raises(engine.Rp3dgError):
        ctx.narrowphase_host(algo, pairs, A.HostContacts(pairs.n, 0))
    # a pair naming a shape outside the table: not colliding, error bit set
    oob = pairs.slice(0, 2)
    oob.shape2[1] = 10_000
    assert ctx.device_errors(clear=True) == 0
    out = ctx.narrowphase_host(algo, oob)
    assert out.is_colliding[1] == 0 and out.nb_contacts[1] == 0
    assert ctx.device_errors(clear=True) & 1
    bad = np.array(z["shapes"])
    bad["kind"][0] = 9
    with pytest.raises(engine.Rp3dgError):
        ctx.set_shapes(bad)


def test_full_size_scene_properties(ctx, port_hulls):
    """The full 1,048,576-pair workload: every batch runs on device memory,
    two runs are bit-identical, and a random 3% sample of pairs agrees
    bit-for-bit with the oracle."""
    sc = scenes.narrowphase_scene(seed=1234, hull=edgecases.load_hull())
    assert sc.n_pairs == scenes.TOTAL_PAIRS
    ctx.set_shapes(sc.shapes)
    rng = np.random.default_rng(5)
    for name, (algo, pairs) in sc.batches.items():
        dp = engine.DevicePairs(pairs)
        o1 = engine.DeviceContacts(pairs.n)
        o2 = engine.DeviceContacts(pairs.n)
        ctx.narrowphase_device(algo, dp, o1)
        ctx.narrowphase_device(algo, dp, o2)
        ctx.synchronize()
        h1, h2 = o1.to_host(), o2.to_host()
        assert reflib.compare_contacts(h1, h2, pairs.n) == {k: 0 for k in reflib.compare_contacts(h1, h2, pairs.n)}
        idx = np.sort(rng.choice(pairs.n, size=max(64, pairs.n // 33), replace=False))
        sub = A.HostPairs(pairs.shape1[idx], pairs.shape2[idx], pairs.pos1[idx], pairs.rot1[idx], pairs.pos2[idx],
                          pairs.rot2[idx])
        exp, _ = port_hulls.narrowphase(algo, sc.shapes, sub)
        got = A.HostContacts(len(idx))
        got.is_colliding[:] = h1.is_colliding[idx]
        got.nb_contacts[:] = h1.nb_contacts[idx]
        got.normal_depth[:] = h1.normal_depth[:, idx]
        got.local1[:] = h1.local1[:, idx]
        got.local2[:] = h1.local2[:, idx]
        _assert_same(got, exp, what=name + " sample")
        # contact normals are unit vectors and depths positive
        m = h1.valid_mask()
        nd = h1.normal_depth[m]
        assert np.all(nd[:, 3] > 0)
        assert np.allclose(np.linalg.norm(nd[:, :3], axis=1), 1.0, atol=1e-4)


def test_grazing_capsule_clip_matches_oracle(ctx, port_hulls):
    """Capsules on a box face almost parallel to one of its edges, crossing
    the edge's side plane at a grazing angle: clipSegmentWithPlanes keeps one
    vertex and its next plane reads the array's stale second slot (the
    previous second vertex); the GPU reproduces it."""
    sh = edgecases.shape_table()
    ctx.set_shapes(sh)
    b = edgecases.grazing_capsule_batch(4096, seed=5)
    exp, _ = port_hulls.narrowphase(A.ALGO_CAPSULE_VS_CONVEX_POLYHEDRON, sh, b.slice(0, b.n))
    got = ctx.narrowphase_host(A.ALGO_CAPSULE_VS_CONVEX_POLYHEDRON, b.slice(0, b.n))
    _assert_same(got, exp, what="grazing capsules")
    if reflib.have_ref("f32"):
        ref = reflib.RefEngine("f32")
        a, _ = ref.narrowphase(A.ALGO_CAPSULE_VS_CONVEX_POLYHEDRON, _remap_meshes(sh, _register_hulls(ref)),
                               b.slice(0, b.n))
        _assert_same(got, a, what="grazing capsules vs reference")


def test_narrowphase_input_small_slots_and_empty_batches(ctx):
    """rp3dg_narrowphase_input_host with batches of 4 and 8 contact slots per
    pair, an empty batch and a batch with report_contacts off for half its
    pairs: each batch's results equal those of rp3dg_narrowphase_host on it
    (two calls, so the second copies the expected number of contacts)."""
    sc = scenes.narrowphase_scene(total_pairs=7 * 3000, seed=77, hull=edgecases.load_hull())
    ctx.set_shapes(sc.shapes)
    for call in range(2):
        batches, refs = [], []
        for k, (name, (algo, pairs)) in enumerate(sc.batches.items()):
            n = 0 if k == 2 else pairs.n
            pr = pairs.slice(0, n)
            if k == 4:
                pr.report = (np.arange(n) % 2).astype(np.uint8)
            mc = (4, 8, 16)[k % 3]
            exp = ctx.narrowphase_host(algo, pr.slice(0, n), A.HostContacts(n, mc)) if n else None
            batches.append((algo, pr, A.HostContacts(n, mc)))
            refs.append(exp)
        got = ctx.narrowphase_input_host(batches)
        for (algo, pr, _), g, exp in zip(batches, got, refs):
            if exp is None:
                assert g.n == 0
                continue
            _assert_same(g, exp, what=f"algo {algo} slots {g.max_contacts} call {call}")


@pytest.mark.parametrize("pinned", [False, True])
def test_narrowphase_input_matches_per_batch_calls(ctx, pinned):
    """rp3dg_narrowphase_input_host (all batches overlapped, contacts packed
    on the device and scattered into the outputs on the host) gives, batch by
    batch, the results and caches of rp3dg_narrowphase_host, on three frames
    (fresh caches, then moved poses with the previous frame's caches): the
    first call copies each batch's contacts back once their count is known,
    the later ones copy the expected number with the flags and fall back to
    the first way for a batch with more contacts than expected."""
    import torch
    sc = scenes.narrowphase_scene(total_pairs=7 * 6000, seed=321, hull=edgecases.load_hull())
    ctx.set_shapes(sc.shapes)
    rng = np.random.default_rng(4)

    def pin(a):
        a = np.ascontiguousarray(a)
        if not pinned:
            return a.copy()
        b = torch.from_numpy(a.view(np.uint8).reshape(-1)).pin_memory().numpy()
        return b.view(a.dtype).reshape(a.shape)

    def outs_for(n):
        o = A.HostContacts(n)
        for f in ("is_colliding", "nb_contacts", "normal_depth", "local1", "local2"):
            setattr(o, f, pin(getattr(o, f)))
        return o

    frames = []
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        frames.append((name, algo, pairs))
    for frame in range(3):
        ref, batches = [], []
        for name, algo, pairs in frames:
            pr = pairs.slice(0, pairs.n)
            pb = A.HostPairs(pin(pairs.shape1), pin(pairs.shape2), pin(pairs.pos1), pin(pairs.rot1),
                             pin(pairs.pos2), pin(pairs.rot2), None, pin(pairs.cache))
            ref.append((ctx.narrowphase_host(algo, pr), pr.cache))
            batches.append((algo, pb, outs_for(pairs.n)))
        got = ctx.narrowphase_input_host(batches)
        for (name, _, _), (exp, cache_exp), g, (_, pb, _) in zip(frames, ref, got, batches):
            _assert_same(g, exp, pb.cache, cache_exp, f"{name} frame {frame + 1} pinned={pinned}")
        # the next frame: moved poses, the caches the reference's collision
        # detection leaves
        frames = [(name, algo, reflib.perturb_pairs(pairs, rng)) for name, algo, pairs in frames]
        for k, (name, algo, pairs) in enumerate(frames):
            pairs.cache = reflib.next_frame_cache(ref[k][1], ref[k][0])
