"""The reference's raycast (oracle/_ref) against the known answers of its
own raycast test (tests/golden/raycast_known.json), on the CPU."""
import numpy as np
import pytest

import rayio
import reflib
from reactphysics3d_b200 import _abi as A

SHAPES = ("box", "sphere", "capsule", "convex_mesh", "concave_mesh", "heightfield")


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built (make -C oracle ref)")
@pytest.mark.parametrize("shape", SHAPES)
def test_reference_raycast_reproduces_known_answers(shape):
    k = rayio.load_known()
    cases = k["cases"][shape]
    assert len(cases) >= 15
    sc, to_world = rayio.known_world(k, shape)
    r = reflib.RefScene(sc)
    hits, counts = r.raycast(rayio.known_rays(cases, to_world), A.RAYCAST_ALL, 4)
    rayio.check_known(cases, to_world, hits, counts)


def test_known_answer_fixture_covers_hits_and_misses():
    k = rayio.load_known()
    for shape in SHAPES:
        cs = k["cases"][shape]
        assert any(c["hit"] for c in cs) and any(not c["hit"] for c in cs), shape
        assert any("fraction" in c and "hit_point" in c for c in cs), shape
        assert any(c["max_fraction"] != 1.0 for c in cs), shape
