"""Batched world raycast on the GPU (rp3dg_world_raycast, the drop-in for
PhysicsWorld::raycast) against the reference float build: for every ray the
number of hits the callback receives and each reported hit (point, normal,
fraction, body, collider) must be bit-identical, in the CLOSEST, ANY and ALL
callback modes; and the known answers of the reference's own raycast test
must hold."""
import numpy as np
import pytest

import rayio
import reflib
import worldio
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes

pytestmark = pytest.mark.gpu
MODES = ((A.RAYCAST_CLOSEST, 1), (A.RAYCAST_ANY, 1), (A.RAYCAST_ALL, 6))
needs_ref = pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    yield c
    c.close()


def _compare(w, r, rays, world=0):
    for mode, k in MODES:
        got = w.raycast(rays, mode, k, world=world)
        exp = r.raycast(rays, mode, k)
        assert rayio.same_hits(got, exp), mode
    return got


@needs_ref
@pytest.mark.parametrize("shape", ("box", "sphere", "capsule", "convex_mesh", "concave_mesh", "heightfield"))
def test_raycast_known_answers(ctx, shape):
    """The reference test's rays against one shape: bit-identical to the
    reference in all modes, and its expected hits, fractions and points."""
    k = rayio.load_known()
    cases = k["cases"][shape]
    sc, to_world = rayio.known_world(k, shape)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    rays = rayio.known_rays(cases, to_world)
    hits, counts = _compare(w, r, rays)
    rayio.check_known(cases, to_world, hits, counts)
    w.close()


@needs_ref
def test_raycast_hull_world_matches_reference(ctx):
    """Hulls (two scales), boxes, spheres and capsules, before and after they
    fall and settle: 20000 rays per check, category masks 0xFFFF, 1 and 2,
    and a maxFraction below 1 for a third of the rays."""
    sc = scenes.hull_world(6, 3, 6, seed=19)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    for steps, advance in ((0, 45), (45, 105), (150, 0)):
        rays = scenes.world_rays(20000, (-6, -0.5, -6), (6, 6, 6), seed=steps, masks=(0xFFFF, 1, 2))
        rays["max_fraction"][::3] = np.float32(0.6)
        hits, counts = _compare(w, r, rays)
        assert (counts > 0).sum() > 5000
        kinds = sc.shapes["kind"][sc.colliders["shape"][hits[counts > 0, 0]["collider"]]]
        assert set(np.unique(kinds)) >= {A.SHAPE_BOX, A.SHAPE_SPHERE, A.SHAPE_CAPSULE, A.SHAPE_CONVEX_MESH}
        if advance:
            w.update(float(worldio.DT), advance)
            r.update(float(worldio.DT), advance)


@needs_ref
def test_raycast_terrain_matches_reference(ctx):
    """A height-field terrain on a tilted, shifted body with bodies resting on
    it: rays straight down walk one cell, slanted rays walk the grid."""
    sc = scenes.heightfield_world(n_bodies=300, cols=40, rows=33, cell=1.25, y_scale=0.8, seed=23,
                                  terrain_position=(0.5, -0.3, 0.25),
                                  terrain_orientation=(0.0499792, 0.0, 0.0299875, 0.9983002))
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    w.update(float(worldio.DT), 90)
    r.update(float(worldio.DT), 90)
    lo, hi = (-25, -3, -21), (25, 8, 21)
    down = scenes.world_rays(10000, lo, hi, seed=3, down=1.0)
    down["point2"][:, 0] = down["point1"][:, 0]          # exactly vertical: one cell each
    down["point2"][:, 2] = down["point1"][:, 2]
    slanted = scenes.world_rays(10000, lo, hi, seed=4, down=0.0)
    for rays, min_hits in ((down, 8000), (slanted, 1000)):
        hits, counts = _compare(w, r, rays)
        assert (counts > 0).sum() > min_hits, (counts > 0).sum()
        assert (hits[counts > 0, 0]["flags"] == 0).all()
        hf = sc.colliders["shape"][hits[counts > 0, 0]["collider"]]
        assert (sc.shapes["kind"][hf] == A.SHAPE_HEIGHTFIELD).any()


@needs_ref
def test_raycast_mixed_world_with_sleep_and_filters(ctx):
    """Sleeping and kinematic bodies, category filters: the mixed world after
    it settles, rays with masks 0xFFFF, 1, 2, 4 and 0 (no collider)."""
    sc = scenes.mixed_world(5, 4, 5, seed=5)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    w.update(float(worldio.DT), 200)
    r.update(float(worldio.DT), 200)
    assert w.bodies()[4].sum() > 0
    rays = scenes.world_rays(20000, (-5, -0.5, -5), (5, 5, 5), seed=7, masks=(0xFFFF, 1, 2, 4, 0))
    hits, counts = _compare(w, r, rays)
    assert (counts[4::5] == 0).all()


@needs_ref
def test_raycast_edge_rays(ctx):
    """Zero-length rays, rays starting inside shapes, axis-parallel rays
    (direction components exactly zero), maxFraction 0, 0.25 and 3."""
    sc = scenes.hull_world(4, 2, 4, seed=21)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    w.update(float(worldio.DT), 60)
    r.update(float(worldio.DT), 60)
    rng = np.random.default_rng(5)
    centres = w.bodies()[0][1:]
    n = len(centres)
    rays = A.rays(6 * n)
    p = centres.astype(np.float32)
    rays["point1"][:n] = p
    rays["point2"][:n] = p                                          # zero length, at a centre
    rays["point1"][n:2 * n] = p
    rays["point2"][n:2 * n] = p + rng.uniform(-3, 3, (n, 3)).astype(np.float32)   # from inside
    for a in range(3):                                              # parallel to x, y, z
        s = slice((2 + a) * n, (3 + a) * n)
        q = p + rng.uniform(-0.3, 0.3, (n, 3)).astype(np.float32)
        rays["point1"][s] = q
        rays["point2"][s] = q
        rays["point1"][s, a] -= np.float32(8.0)
        rays["point2"][s, a] += np.float32(8.0)
    rays["point1"][5 * n:] = p + np.float32([0.0, 6.0, 0.0])
    rays["point2"][5 * n:] = p - np.float32([0.0, 6.0, 0.0])
    for mf in (0.0, 0.25, 1.0, 3.0):
        rays["max_fraction"] = np.float32(mf)
        hits, counts = _compare(w, r, rays)
        if mf == 1.0:
            assert (counts[2 * n:] > 0).sum() > n


@needs_ref
def test_raycast_group_worlds(ctx):
    """Each world of a group is cast against its own tree."""
    parts = [scenes.hull_world(3, 2, 3, seed=31), scenes.mixed_world(3, 3, 3, seed=32, variety=False)]
    shapes, merged = scenes.merge_shapes(parts)
    g = engine.WorldGroup(ctx, merged, shapes)
    refs = [reflib.RefScene(s) for s in parts]
    g.update(float(worldio.DT), 30)
    for rr in refs:
        rr.update(float(worldio.DT), 30)
    rays = scenes.world_rays(8000, (-4, -0.5, -4), (4, 4, 4), seed=9)
    for k, rr in enumerate(refs):
        _compare(g, rr, rays, world=k)
    g.close()


def test_raycast_rejects_bad_arguments(ctx):
    sc = scenes.box_pile(2, 2, 2)
    w = engine.World(ctx, sc)
    rays = A.rays(4)
    with pytest.raises(engine.Rp3dgError):
        w.raycast(rays, mode=7)
    with pytest.raises(engine.Rp3dgError):
        w.raycast(rays, world=3)
    hits, counts = w.raycast(A.rays(0))
    assert len(counts) == 0
    w.close()
