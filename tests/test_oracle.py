"""The C restatement (oracle/rp3d_oracle.c) against the reference engine's own
outputs: committed golden fixtures always, the live reference build
(oracle/_ref) when it is present.  Bit-exact, every field."""
import numpy as np
import pytest

import edgecases
import goldenio
import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import scenes

GOLDEN = reflib.ROOT + "/tests/golden/"


def _assert_same(got, exp, cache_got=None, cache_exp=None, what=""):
    mism = reflib.compare_contacts(got, exp, exp.n)
    assert all(v == 0 for v in mism.values()), (what, mism)
    if cache_exp is not None:
        a = cache_got.view(np.uint8).reshape(-1, 16)
        b = cache_exp.view(np.uint8).reshape(-1, 16)
        assert np.array_equal(a, b), (what, "cache", np.argwhere(a != b)[:5])


def _register_hulls(engine):
    v, f = edgecases.load_hull()
    m = engine.create_convex_mesh(v, f)
    engine.create_convex_mesh_shape(m)
    engine.create_convex_mesh_shape(m, edgecases.HULL_SCALE)


@pytest.fixture(scope="module")
def port_hulls(port):
    port.lib.rp3do_reset()
    _register_hulls(port)
    return port


@pytest.mark.parametrize("fixture", ["np_scene.npz", "np_edge.npz"])
def test_port_matches_golden(port_hulls, fixture):
    z = np.load(GOLDEN + fixture)
    shapes = z["shapes"]
    prefixes = goldenio.case_prefixes(z)
    assert prefixes
    for pre in prefixes:
        algo, clip, pairs, exp, cache_exp = goldenio.unpack_case(z, pre)
        got, _ = port_hulls.narrowphase(algo, shapes, pairs, out=A.HostContacts(pairs.n, exp.max_contacts), clip=clip)
        _assert_same(got, exp, pairs.cache, cache_exp, pre)


def test_port_mesh_tables_match_golden_hull(port_hulls):
    t = port_hulls.mesh_tables(0)
    assert t["half_edges"].shape == (240, 4)
    he = t["half_edges"]
    # half-edge invariants: twins pair up, next stays on the face
    assert np.all(he[he[:, 1], 1] == np.arange(len(he)))
    assert np.all(he[he[:, 3], 2] == he[:, 2])
    assert np.allclose(np.linalg.norm(t["face_normals"], axis=1), 1.0, atol=1e-6)


needs_ref = pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build oracle/_ref not present")


@needs_ref
def test_port_mesh_tables_match_reference(port_hulls):
    ref = reflib.RefEngine("f32")
    _register_hulls(ref)
    for inst in (0, 1):
        a, b = port_hulls.mesh_tables(inst), ref.mesh_tables(inst)
        assert np.array_equal(a["half_edges"], b["half_edges"])
        assert np.array_equal(a["face_edge"], b["face_edge"])
        assert np.array_equal(a["face_normals"].view(np.uint32), b["face_normals"].view(np.uint32))
        assert np.array_equal(a["centroid"].view(np.uint32), b["centroid"].view(np.uint32))


@needs_ref
@pytest.mark.parametrize("seed", [21, 22])
def test_port_matches_reference_random(port_hulls, seed):
    ref = reflib.RefEngine("f32")
    _register_hulls(ref)
    sc = scenes.narrowphase_scene(total_pairs=7 * 1500, seed=seed, hull=edgecases.load_hull())
    rng = np.random.default_rng(seed)
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        pr, pp = pairs.slice(0, pairs.n), pairs.slice(0, pairs.n)
        a, _ = ref.narrowphase(algo, sc.shapes, pr)
        b, _ = port_hulls.narrowphase(algo, sc.shapes, pp)
        _assert_same(b, a, pp.cache, pr.cache, name + " fresh")
        nxt = reflib.perturb_pairs(pr, rng)
        nxt.cache = reflib.next_frame_cache(pr.cache, a)
        pr2, pp2 = nxt.slice(0, nxt.n), nxt.slice(0, nxt.n)
        a2, _ = ref.narrowphase(algo, sc.shapes, pr2)
        b2, _ = port_hulls.narrowphase(algo, sc.shapes, pp2)
        _assert_same(b2, a2, pp2.cache, pr2.cache, name + " coherent")


def test_planted_mistake_is_caught(port_hulls):
    """The comparison must notice a one-ulp change in a single contact."""
    z = np.load(GOLDEN + "np_scene.npz")
    algo, clip, pairs, exp, _ = goldenio.unpack_case(z, "box_box_a_")
    got, _ = port_hulls.narrowphase(algo, z["shapes"], pairs, clip=clip)
    k = int(np.argmax(got.nb_contacts > 0))
    got.normal_depth[0, k, 3] = np.nextafter(got.normal_depth[0, k, 3], np.float32(np.inf))
    assert reflib.compare_contacts(got, exp, exp.n)["normal_depth"] == 1


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build oracle/_ref not present")
def test_grazing_capsule_clip_matches_reference(port):
    """clipSegmentWithPlanes' one-vertex branch (segment nearly parallel to a
    side plane): the next plane reads the array's stale second slot."""
    ref = reflib.RefEngine("f32")
    sh = edgecases.shape_table()
    ids = []
    for e in (ref, port):
        if e is port:
            port.lib.rp3do_reset()
        v, f = edgecases.load_hull()
        m = e.create_convex_mesh(v, f)
        ids.append((e.create_convex_mesh_shape(m), e.create_convex_mesh_shape(m, edgecases.HULL_SCALE)))
    b = edgecases.grazing_capsule_batch(4096, seed=5)
    a, _ = ref.narrowphase(A.ALGO_CAPSULE_VS_CONVEX_POLYHEDRON, sh, b.slice(0, b.n))
    c, _ = port.narrowphase(A.ALGO_CAPSULE_VS_CONVEX_POLYHEDRON, sh, b.slice(0, b.n))
    assert reflib.compare_contacts(c, a, b.n) == {k: 0 for k in ("is_colliding", "nb_contacts", "normal_depth",
                                                                  "local1", "local2")}
    assert (a.nb_contacts == 1).sum() > 100 and (a.nb_contacts == 2).sum() > 100
