"""World step fixture checks on the CPU: the reference engine (built from its
sources into oracle/_ref) reproduces the golden world trajectories, and the
scene generators are deterministic."""
import os

import numpy as np
import pytest

import reflib
import worldio
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "world.npz")


def fixture(name):
    z = np.load(GOLDEN)
    return {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built (make -C oracle ref)")
@pytest.mark.parametrize("name", list(worldio.WORLD_CASES))
def test_reference_reproduces_world_fixture(name):
    sc, steps, every = worldio.make_scene(name)
    got = worldio.trajectory(reflib.RefScene(sc), steps, every, worldio.DRIVERS.get(name))
    exp = fixture(name)
    assert worldio.first_mismatch(got, exp) is None
    for k in ("ckpt_pos", "ckpt_ori", "ckpt_lv", "ckpt_av", "ckpt_sleep"):
        assert np.array_equal(got[k], exp[k]), k


def test_world_fixture_exercises_sleeping_and_contacts():
    for name in ("pile125", "mixed100"):
        f = fixture(name)
        assert f["ckpt_sleep"][-1].sum() > 0, name        # some bodies fall asleep
        assert f["man_n"].max() > 50 and f["pt_n"].max() > f["man_n"].max(), name


def test_scene_generators_are_deterministic():
    a, b = scenes.box_pile(4, 3, 4, seed=9), scenes.box_pile(4, 3, 4, seed=9)
    for f in ("shapes", "bodies", "colliders"):
        assert getattr(a, f).tobytes() == getattr(b, f).tobytes()
    assert a.bodies.dtype == A.BODY_DESC_DTYPE and a.colliders.dtype == A.COLLIDER_DESC_DTYPE
    m = scenes.mixed_world(seed=4)
    assert set(np.unique(m.shapes["kind"][1:])) == {A.SHAPE_SPHERE, A.SHAPE_CAPSULE, A.SHAPE_BOX}
    assert (m.bodies["type"] == A.BODY_KINEMATIC).any() and m.bodies["type"][0] == A.BODY_STATIC
