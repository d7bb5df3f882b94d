"""DebugRenderer as headless device buffers (rp3dg_world_get_debug_primitives):
after every update the lines and triangles of DebugRenderer::onContact and
computeDebugRenderingPrimitives (src/utils/DebugRenderer.cpp:482-560) are
bit-identical to the reference engine's getLinesArray / getTrianglesArray,
on worlds of boxes, spheres and capsules, of convex meshes, on a height
field and on a concave mesh; with every item shown on every body, and with
a subset of the items on a subset of the bodies switched on, changed and
off between updates."""
import numpy as np
import pytest

import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build absent")]
DT = float(np.float32(1.0 / 60.0))


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    yield c
    c.close()


def _check(w, r, tag):
    lw, tw = w.debug_primitives()
    lr, tr = r.debug_primitives()
    assert (len(lw), len(tw)) == (len(lr), len(tr)), (tag, len(lw), len(lr), len(tw), len(tr))
    assert lw.tobytes() == lr.tobytes(), (tag, "lines", _first_diff(lw, lr))
    assert tw.tobytes() == tr.tobytes(), (tag, "triangles", _first_diff(tw, tr))
    return lw, tw


def _first_diff(a, b):
    for k in range(min(len(a), len(b))):
        if a[k].tobytes() != b[k].tobytes():
            return k, a[k], b[k]
    return None


SCENES = [
    ("mixed", lambda: scenes.mixed_world(nx=3, ny=3, nz=3, seed=5, variety=True), 90),
    ("hulls", lambda: scenes.hull_world(3, 2, 3, seed=44), 90),
    ("terrain", lambda: scenes.heightfield_world(n_bodies=40, cols=12, rows=12, seed=45), 90),
    ("concave_mesh", lambda: scenes.concave_mesh_world(n_bodies=40, cols=10, rows=10, seed=46, scale=(1.2, 1.0, 0.9)),
     90),
]


@pytest.mark.parametrize("name,make,steps", SCENES)
def test_debug_primitives_match_reference(ctx, name, make, steps):
    sc = make()
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    for x in (w, r):
        x.set_debug_rendering(A.DEBUG_ALL)
        x.set_body_debug(-1, True)
    colors = set()
    for s in range(steps):
        w.update(DT)
        r.update(DT)
        lw, tw = _check(w, r, (name, s))
        colors |= set(lw["color1"].tolist()) | set(tw["color1"].tolist())
    # every item showed up: AABBs, fat AABBs, shapes, contact points and normals, shape normals
    assert colors == {0xff00ff, 0xffff00, 0x00ff00, 0xff0000, 0xffffff, 0x0000ff}, (name, sorted(colors))
    w.close()


def test_debug_items_and_bodies_switched(ctx):
    sc = scenes.mixed_world(nx=3, ny=2, nz=3, seed=8, variety=False)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    nb = len(sc.bodies)
    plan = {
        5: A.DEBUG_COLLIDER_AABB | A.DEBUG_CONTACT_NORMAL,
        25: A.DEBUG_COLLISION_SHAPE_NORMAL | A.DEBUG_COLLIDER_BROADPHASE_AABB | A.DEBUG_CONTACT_POINT,
        45: A.DEBUG_COLLISION_SHAPE,
        60: 0,   # off: the renderer is no longer reset, the last primitives stay
        70: A.DEBUG_ALL,
    }
    for b in range(0, nb, 3):
        for x in (w, r):
            x.set_body_debug(b, True)
    for s in range(80):
        if s in plan:
            for x in (w, r):
                x.set_debug_rendering(plan[s])
        if s == 50:
            for x in (w, r):
                x.set_body_debug(1, True)
                x.set_body_debug(0, False)
        w.update(DT)
        r.update(DT)
        _check(w, r, s)
    w.close()
