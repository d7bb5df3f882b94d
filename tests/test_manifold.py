"""Contact-manifold reduction, CPU side: the C restatement
(rp3do_reduce_contacts) against the reference's reduceContactPoints +
removeDuplicatedContactPointsInManifold, through the committed fixture and,
when oracle/_ref is built, live on a seeded scene."""
import numpy as np
import pytest

import edgecases
import goldenio
import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import scenes

GOLDEN = reflib.ROOT + "/tests/golden/np_manifold.npz"


def assert_reduced_equal(got, exp, kept_got=None, kept_exp=None, what=""):
    """Bit-exact over the kept slots; slots past nb_contacts are not compared."""
    assert np.array_equal(got.is_colliding, exp.is_colliding), what
    assert np.array_equal(got.nb_contacts, exp.nb_contacts), (what, np.flatnonzero(got.nb_contacts != exp.nb_contacts)[:5])
    m = exp.valid_mask()
    for f in ("normal_depth", "local1", "local2"):
        a = getattr(got, f)[: exp.max_contacts][m].view(np.uint32)
        b = getattr(exp, f)[m].view(np.uint32)
        assert np.array_equal(a, b), (what, f)
    if kept_exp is not None:
        assert np.array_equal(kept_got, kept_exp), (what, "kept", np.argwhere(kept_got != kept_exp)[:5])


@pytest.fixture(scope="module")
def manifold():
    return np.load(GOLDEN)


def test_fixture_shape(manifold):
    groups = goldenio.manifold_groups(manifold)
    assert "box_box" in groups and "hull_box" in groups and "synthetic" in groups
    _, raw, red, kept = goldenio.unpack_manifold(manifold, "box_box")
    assert (raw.nb_contacts > 4).sum() > 50
    assert red.nb_contacts.max() <= 4
    _, raw, red, kept = goldenio.unpack_manifold(manifold, "synthetic")
    assert (np.minimum(raw.nb_contacts, 4) != red.nb_contacts).sum() > 50  # de-duplications


def test_oracle_matches_reference_fixture(port, manifold):
    for name in goldenio.manifold_groups(manifold):
        pairs, raw, red, kept = goldenio.unpack_manifold(manifold, name)
        got = reflib.copy_contacts(raw)
        k = reflib.reduce_contacts(port.lib, "rp3do_reduce_contacts", pairs, got)
        assert_reduced_equal(got, red, k, kept, name)


def test_reduced_manifold_properties(port, manifold):
    """Kept points are distinct raw slots, at most 4, at least 0.01 apart."""
    pairs, raw, red, kept = goldenio.unpack_manifold(manifold, "synthetic")
    got = reflib.copy_contacts(raw)
    k = reflib.reduce_contacts(port.lib, "rp3do_reduce_contacts", pairs, got)
    for i in range(pairs.n):
        m = int(got.nb_contacts[i])
        ks = k[i, :m]
        assert np.all(k[i, m:] == 255) and len(set(ks.tolist())) == m and np.all(ks < raw.nb_contacts[i])
        assert np.array_equal(got.local1[:m, i], raw.local1[ks, i])
        if got.is_colliding[i] and m > 1:
            p = got.local1[:m, i, :3]
            d2 = ((p[:, None] - p[None]) ** 2).sum(-1) + np.eye(m)
            assert d2.min() >= np.float32(0.01) ** 2 * 0.999


def test_empty_batch(port):
    z = np.zeros(0, np.int32)
    pairs = A.HostPairs(z, z, np.zeros((0, 4)), np.zeros((0, 4)), np.zeros((0, 4)), np.zeros((0, 4)))
    k = reflib.reduce_contacts(port.lib, "rp3do_reduce_contacts", pairs, A.HostContacts(0))
    assert k.shape == (0, 4)


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build oracle/_ref not present")
def test_oracle_matches_reference_live(port):
    ref = reflib.RefEngine("f32")
    v, f = edgecases.load_hull()
    m = ref.create_convex_mesh(v, f)             # same instance numbering as the other reference tests:
    ref.create_convex_mesh_shape(m)              # 0 = hull, 1 = scaled hull
    ref.create_convex_mesh_shape(m, edgecases.HULL_SCALE)
    sc = scenes.narrowphase_scene(total_pairs=7 * 4096, seed=404, hull=(v, f))
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        p0 = pairs.slice(0, pairs.n)
        out, _ = ref.narrowphase(algo, sc.shapes, p0)       # p0.cache: the narrow phase's records
        a, b = reflib.copy_contacts(out), reflib.copy_contacts(out)
        pa, pb = p0.slice(0, p0.n), p0.slice(0, p0.n)
        ka = reflib.reduce_contacts(ref.lib, "ref_reduce_contacts", pa, a)
        kb = reflib.reduce_contacts(port.lib, "rp3do_reduce_contacts", pb, b)
        assert_reduced_equal(b, a, kb, ka, name)
        # the last-frame records: valid, and remembering this frame's result
        assert np.array_equal(pa.cache.view(np.uint8), pb.cache.view(np.uint8)), name
        assert np.array_equal(pb.cache, reflib.next_frame_cache(p0.cache, out)), name
