"""Trigger colliders in the world step (Collider::setIsTrigger): their pairs
are tested without contact points, colliding ones become contact pairs that
no island takes, and EventListener::onTrigger reports them (OverlapStart /
Stay / Exit) while onContact leaves them out.  Live against the reference
engine: every step's pairs, contact manifolds, contact events, trigger
events and final states bit-identical, on a mixed world and on a
height-field world (convex triggers against the terrain's triangles)."""
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


def _same(a, b):
    return all(np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8)) for x, y in zip(a, b))


@pytest.mark.parametrize("name,scene,steps", [
    ("mixed", lambda: scenes.with_triggers(scenes.mixed_world(nx=4, ny=3, nz=4, seed=21, variety=False)), 180),
    ("terrain", lambda: scenes.with_triggers(scenes.heightfield_world(n_bodies=60, cols=24, rows=24, seed=11),
                                             every=4, zones=((0.0, 3.0, 0.0, 3.0, 1.0, 3.0),)), 180),
])
def test_triggers_match_reference(ctx, name, scene, steps):
    sc = scene()
    assert (sc.colliders["flags"] & A.COLLIDER_TRIGGER).sum() >= 3
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    n_trig = 0
    kinds = set()
    for s in range(steps):
        w.update(DT)
        r.update(DT)
        assert np.array_equal(w.pairs(), r.pairs()), (name, s)
        assert _same(w.contacts(), r.contacts()), (name, s)
        te, tr = w.trigger_events(), r.trigger_events()
        assert np.array_equal(te, tr), (name, s, te[:4], tr[:4])
        ce, cr = w.contact_events(), r.contact_events()
        assert np.array_equal(ce[0], cr[0]), (name, s)
        n_trig += len(te)
        kinds |= set(te["type"].tolist())
    assert _same(w.bodies(), r.bodies()), name
    # overlaps started, stayed and ended
    assert n_trig > 0 and kinds == {A.CONTACT_START, A.CONTACT_STAY, A.CONTACT_EXIT}, (n_trig, kinds)
    w.close()
