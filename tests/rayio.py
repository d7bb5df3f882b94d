"""Raycast test helpers: the known-answer worlds of the reference's raycast
test (tests/golden/raycast_known.json) and the comparison of hit records."""
import json
import os

import numpy as np

from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import scenes

KNOWN = os.path.join(os.path.dirname(__file__), "golden", "raycast_known.json")


def euler_quaternion(ax, ay, az):
    """Quaternion::fromEulerAngles (Quaternion.cpp:207-233), float64."""
    sx, cx = np.sin(0.5 * ax), np.cos(0.5 * ax)
    sy, cy = np.sin(0.5 * ay), np.cos(0.5 * ay)
    sz, cz = np.sin(0.5 * az), np.cos(0.5 * az)
    q = np.array([sx * cy * cz - cx * sy * sz, cx * sy * cz + sx * cy * sz,
                  cx * cy * sz - sx * sy * cz, cx * cy * cz + sx * sy * sz])
    return q / np.linalg.norm(q)


def _apply(pos, q, p):
    return scenes._rotate(q, np.atleast_2d(p)) + np.asarray(pos)


def load_known():
    with open(KNOWN) as fh:
        return json.load(fh)


def known_world(k, shape):
    """The world of one shape of the reference test: one static body at the
    test's body transform with the shape at the test's shape transform; the
    local-to-world map of the shape's space (float64)."""
    bq = euler_quaternion(*(np.pi * np.array(k["body_euler_pi"])))
    sq = euler_quaternion(*(np.pi * np.array(k["shape_euler_pi"])))
    shapes = np.zeros(1, A.SHAPE_DTYPE)
    shapes["mesh"] = -1
    hfs, cms, ccs = [], [], []
    if shape == "box":
        shapes[0]["kind"] = A.SHAPE_BOX
        shapes[0]["params"][:3] = k["box_half_extents"]
    elif shape == "sphere":
        shapes[0]["kind"] = A.SHAPE_SPHERE
        shapes[0]["params"][0] = k["sphere_radius"]
    elif shape == "capsule":
        shapes[0]["kind"] = A.SHAPE_CAPSULE
        r, h = k["capsule"]
        shapes[0]["params"][:2] = (r, 0.5 * h)
    elif shape == "convex_mesh":
        shapes[0]["kind"] = A.SHAPE_CONVEX_MESH
        shapes[0]["mesh"] = 0
        cms = [(np.array(k["convex_vertices"], np.float32), k["convex_faces"], (1.0, 1.0, 1.0))]
    elif shape == "concave_mesh":
        shapes[0]["kind"] = A.SHAPE_CONCAVE_MESH
        shapes[0]["mesh"] = 0
        ccs = [(np.array(k["concave_vertices"], np.float32), np.array(k["concave_triangles"], np.uint32), None,
                (1.0, 1.0, 1.0))]
    else:
        hf = k["heightfield"]
        shapes[0]["kind"] = A.SHAPE_HEIGHTFIELD
        shapes[0]["mesh"] = 0
        hfs = [(np.full((hf["rows"], hf["columns"]), hf["height"], np.float32), (1.0, 1.0, 1.0))]
    bodies = A.body_descs(1)
    bodies[0]["type"] = A.BODY_STATIC
    bodies[0]["position"] = np.float32(k["body_position"])
    bodies[0]["orientation"] = bq.astype(np.float32)
    colliders = A.collider_descs(1)
    colliders[0]["position"] = np.float32(k["shape_position"])
    colliders[0]["orientation"] = sq.astype(np.float32)
    sc = scenes.WorldScene(A.default_world_settings(), shapes, bodies, colliders, f"raycast {shape}",
                           heightfields=hfs, convex_meshes=cms, concave_meshes=ccs)
    bq32, sq32 = bodies[0]["orientation"].astype(np.float64), colliders[0]["orientation"].astype(np.float64)

    def to_world(p):
        return _apply(bodies[0]["position"].astype(np.float64), bq32,
                      _apply(colliders[0]["position"].astype(np.float64), sq32, p))
    return sc, to_world


def known_rays(cases, to_world):
    r = A.rays(len(cases))
    r["point1"] = np.concatenate([to_world(c["p1"]) for c in cases]).astype(np.float32)
    r["point2"] = np.concatenate([to_world(c["p2"]) for c in cases]).astype(np.float32)
    r["max_fraction"] = np.array([c["max_fraction"] for c in cases], np.float32)
    return r


def check_known(cases, to_world, hits, counts, eps=1e-4):
    """The reference test's expectations (epsilon 0.0001): hit or miss, and
    the hit fraction and hit point where the test checks them."""
    for c, h, n in zip(cases, hits, counts):
        assert (n > 0) == c["hit"], (c["ray"], c["max_fraction"])
        if "fraction" in c:
            assert abs(float(h[0]["hit_fraction"]) - c["fraction"]) < eps, c["ray"]
        if "hit_point" in c:
            assert np.abs(h[0]["world_point"] - to_world(c["hit_point"])[0]).max() < eps, c["ray"]


def same_hits(a, b):
    """Bitwise equality of two raycasts' results ((hits, counts) pairs): the
    counts, and every record the counts say is filled."""
    (ha, ca), (hb, cb) = a, b
    if not np.array_equal(ca, cb):
        return False
    k = np.minimum(ca, ha.shape[1])
    mask = np.arange(ha.shape[1])[None, :] < k[:, None]
    return ha[mask].tobytes() == hb[mask].tobytes()
