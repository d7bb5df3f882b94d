"""Concave triangle meshes (TriangleMesh + ConcaveMeshShape) in the world
step, against the reference float build: the mesh as TriangleMesh::init
builds it (degenerate triangles dropped, unused vertices removed,
angle-weighted vertex normals, TriangleMesh.cpp:42-333); convex colliders
falling onto a concave-mesh terrain with every step's pairs, manifolds and
points and the final states bit-identical (the triangles of each convex vs
concave pair from the mesh tree's query, ConcaveMeshShape.cpp:135-175, with
the scaled vertex normals smoothing the contacts); world raycasts against
the mesh (ConcaveMeshShape.cpp:179-274) bit-identical in all callback
modes."""
import numpy as np
import pytest

import rayio
import reflib
import worldio
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build absent")]
DT = float(worldio.DT)


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    yield c
    c.close()


def _bowl():
    """A small closed-top bowl: a ring of 12 x 4 vertices and a centre, its
    triangles wound inwards."""
    vs = [(0.0, -1.0, 0.0)]
    for k in range(1, 5):
        r, y = 0.6 * k, -1.0 + 0.35 * k * k / 4.0
        for s in range(12):
            a = 2 * np.pi * s / 12
            vs.append((r * np.cos(a), y, r * np.sin(a)))
    ts = [(0, 1 + (s + 1) % 12, 1 + s) for s in range(12)]
    for k in range(3):
        for s in range(12):
            a, b = 1 + 12 * k + s, 1 + 12 * k + (s + 1) % 12
            ts += [(a, b, b + 12), (a, b + 12, a + 12)]
    return np.array(vs, np.float32), np.array(ts, np.uint32)


@pytest.mark.parametrize("case", ["terrain", "terrain_normals", "bowl"])
def test_triangle_mesh_matches_reference(ctx, case):
    if case == "bowl":
        v, t = _bowl()
        n = None
    else:
        sc = scenes.concave_mesh_world(n_bodies=1, normals=case == "terrain_normals")
        v, t, n, _ = sc.concave_meshes[0]
    mid = ctx.create_triangle_mesh(v, t, n)
    gv, gn, gt = ctx.triangle_mesh(mid)
    rv, rn, rt = reflib.ref_triangle_mesh(v, t, n)
    assert np.array_equal(gt, rt)
    assert gv.tobytes() == rv.tobytes()
    assert gn.tobytes() == rn.tobytes()
    if case != "bowl":
        assert len(gt) == len(t) - 2 and len(gv) == len(v) - 1   # two degenerate triangles, one unused vertex


def test_triangle_mesh_rejects_bad_input(ctx):
    v, t = _bowl()
    with pytest.raises(engine.Rp3dgError):
        ctx.create_triangle_mesh(v, np.array([[0, 1, 99]], np.uint32))      # index out of range
    with pytest.raises(engine.Rp3dgError):
        ctx.create_triangle_mesh(v, np.array([[0, 0, 1]], np.uint32))       # no triangle left
    with pytest.raises(engine.Rp3dgError):
        ctx.create_concave_mesh_shape(ctx.create_triangle_mesh(v, t), (1.0, 0.0, 1.0))
    sc = scenes.concave_mesh_world(n_bodies=4, cols=6, rows=6)
    bad = scenes.WorldScene(sc.settings, sc.shapes, sc.bodies.copy(), sc.colliders,
                            convex_meshes=sc.convex_meshes, concave_meshes=sc.concave_meshes)
    bad.bodies["type"][0] = A.BODY_DYNAMIC
    with pytest.raises(engine.Rp3dgError):
        engine.World(ctx, bad)          # a concave mesh must be on a static body


WORLDS = [
    ("plain", lambda: scenes.concave_mesh_world(n_bodies=200, cols=18, rows=18, seed=61), 240),
    ("scaled_normals", lambda: scenes.concave_mesh_world(n_bodies=150, cols=14, rows=16, seed=62,
                                                         scale=(1.4, 0.8, 1.2), normals=True,
                                                         terrain_orientation=(0.0499792, 0.0, 0.0299875, 0.9983002)),
     200),
]


@pytest.mark.parametrize("name,make,steps", WORLDS)
def test_concave_world_matches_reference(ctx, name, make, steps):
    sc = make()
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    multi = 0
    for s in range(steps):
        w.update(DT)
        r.update(DT)
        if s < 5 or s % 10 == 9 or s == steps - 1:
            assert np.array_equal(w.pairs(), r.pairs()), (name, s)
            cw, cr = w.contacts(), r.contacts()
            for a, b in zip(cw, cr):
                assert np.array_equal(a, b), (name, s)
            keys = cw[0].astype(np.int64) * 100000 + cw[1]
            multi = max(multi, len(keys) - len(np.unique(keys)))
    for a, b in zip(w.bodies(), r.bodies()):
        assert np.array_equal(a, b), name
    assert w.stats()["narrowphase_tests"] > w.stats()["overlapping_pairs"]   # triangle tests ran
    assert w.bodies()[4].sum() > 0 or name != "plain"                         # bodies come to rest
    w.close()


def test_concave_raycast_matches_reference(ctx):
    sc = scenes.concave_mesh_world(n_bodies=120, cols=16, rows=16, seed=63, scale=(1.25, 0.9, 1.1),
                                   terrain_orientation=(0.0499792, 0.0, 0.0299875, 0.9983002))
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    w.update(DT, 60)
    r.update(DT, 60)
    lo, hi = (-10, -3, -9), (10, 6, 9)
    down = scenes.world_rays(8000, lo, hi, seed=5, down=1.0)
    slanted = scenes.world_rays(8000, lo, hi, seed=6, down=0.0)
    slanted["max_fraction"][::3] = np.float32(0.5)
    for rays in (down, slanted):
        for mode, k in ((A.RAYCAST_CLOSEST, 1), (A.RAYCAST_ANY, 1), (A.RAYCAST_ALL, 6)):
            got = w.raycast(rays, mode, k)
            exp = r.raycast(rays, mode, k)
            assert rayio.same_hits(got, exp), mode
        hits, counts = got
        mesh = sc.colliders["shape"][hits[counts > 0, 0]["collider"]]
        assert (sc.shapes["kind"][mesh] == A.SHAPE_CONCAVE_MESH).sum() > 500
    w.close()
