"""Hand-placed narrow-phase cases: degenerate and boundary configurations of
every algorithm (the inputs only; expected outputs come from the reference
engine and are stored in tests/golden/np_edge.npz)."""
import json
import math
import os

import numpy as np

from reactphysics3d_b200 import _abi as A

HULL_SCALE = (1.5, 0.7, 1.2)
HERE = os.path.dirname(os.path.abspath(__file__))

SPH_A, SPH_B, CAP_A, CAP_B, BOX_A, BOX_B, HULL, HULL_S, GROUND = range(9)


def shape_table():
    sh = np.zeros(9, dtype=A.SHAPE_DTYPE)
    sh["mesh"] = -1
    spec = [(A.SHAPE_SPHERE, (0.5, 0, 0)), (A.SHAPE_SPHERE, (0.8, 0, 0)),
            (A.SHAPE_CAPSULE, (0.3, 0.6, 0)), (A.SHAPE_CAPSULE, (0.25, 1.0, 0)),
            (A.SHAPE_BOX, (1.0, 0.5, 0.75)), (A.SHAPE_BOX, (0.5, 0.5, 0.5)),
            (A.SHAPE_CONVEX_MESH, (0, 0, 0)), (A.SHAPE_CONVEX_MESH, (0, 0, 0)),
            (A.SHAPE_BOX, (5.0, 0.5, 5.0))]
    for i, (k, p) in enumerate(spec):
        sh["kind"][i] = k
        sh["params"][i, :3] = p
    sh["mesh"][HULL] = 0
    sh["mesh"][HULL_S] = 1
    return sh


def qaxis(axis, angle_deg):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    h = math.radians(angle_deg) / 2.0
    return np.array([*(a * math.sin(h)), math.cos(h)], np.float32)


I = np.array([0, 0, 0, 1], np.float32)


def qmul(a, b):
    ax, ay, az, aw = map(float, a)
    bx, by, bz, bw = map(float, b)
    return np.array([aw * bx + bw * ax + ay * bz - az * by, aw * by + bw * ay + az * bx - ax * bz,
                     aw * bz + bw * az + ax * by - ay * bx, aw * bw - ax * bx - ay * by - az * bz], np.float32)


def batch(rows, report=None, cache=False):
    """rows: (shape1, shape2, pos1, rot1, pos2, rot2)"""
    n = len(rows)
    s1 = np.array([r[0] for r in rows], np.int32)
    s2 = np.array([r[1] for r in rows], np.int32)
    p1 = np.zeros((n, 4), np.float32)
    p2 = np.zeros((n, 4), np.float32)
    p1[:, :3] = [r[2] for r in rows]
    p2[:, :3] = [r[4] for r in rows]
    q1 = np.array([r[3] for r in rows], np.float32)
    q2 = np.array([r[5] for r in rows], np.float32)
    return A.HostPairs(s1, s2, p1, q1, p2, q2, report=report, cache=A.fresh_cache(n) if cache else None)


def build():
    sh = shape_table()
    z45 = qaxis((0, 0, 1), 45)
    y45 = qaxis((0, 1, 0), 45)
    x90 = qaxis((1, 0, 0), 90)
    z90 = qaxis((0, 0, 1), 90)
    tilt = qmul(qaxis((1, 0, 0), 30), qaxis((0, 1, 0), 20))
    cases = []
    cases.append(("sphere_sphere", A.ALGO_SPHERE_VS_SPHERE, batch([
        (SPH_A, SPH_B, (1, 2, 3), I, (1, 2, 3), I),                 # coincident centres
        (SPH_A, SPH_B, (0, 0, 0), I, (1e-5, 0, 0), tilt),           # nearly coincident
        (SPH_A, SPH_B, (0, 0, 0), I, (1.3, 0, 0), I),               # exactly touching
        (SPH_A, SPH_B, (0, 0, 0), z45, (1.0, 0.3, -0.2), tilt),     # overlapping
        (SPH_A, SPH_B, (0, 0, 0), I, (2.0, 0, 0), I),               # separated
    ], cache=True), 16))
    cases.append(("sphere_capsule", A.ALGO_SPHERE_VS_CAPSULE, batch([
        (SPH_A, CAP_A, (0, 0.2, 0), I, (0, 0, 0), I),               # centre on the capsule axis
        (SPH_A, CAP_A, (0, 1.2, 0), I, (0, 0, 0), I),               # near the top cap
        (SPH_A, CAP_A, (0.7, 0.1, 0), tilt, (0, 0, 0), z45),        # beside the cylinder
        (SPH_A, CAP_A, (2.0, 0, 0), I, (0, 0, 0), I),               # separated
        (CAP_A, SPH_A, (0, 0, 0), x90, (0.1, 0.2, 0.6), I),         # capsule first
    ], cache=True), 16))
    cases.append(("capsule_capsule", A.ALGO_CAPSULE_VS_CAPSULE, batch([
        (CAP_A, CAP_B, (0.4, 0, 0), I, (0, 0, 0), I),               # parallel side by side
        (CAP_A, CAP_B, (0, 0.3, 0), I, (0, 0, 0), I),               # parallel, same axis
        (CAP_A, CAP_B, (0, 1.8, 0), I, (0, 0, 0), I),               # parallel, end to end
        (CAP_A, CAP_B, (0, 0, 0), z90, (0, 0, 0), I),               # crossing axes (distance 0)
        (CAP_A, CAP_B, (0, 0, 0.4), z90, (0, 0, 0), I),             # crossing, overlapping
        (CAP_A, CAP_B, (0, 0, 1.0), z90, (0, 0, 0), I),             # crossing, separated
        (CAP_A, CAP_B, (0.3, 0.2, 0.1), tilt, (0, 0, 0), z45),      # skew overlapping
    ], cache=True), 16))
    cases.append(("sphere_poly", A.ALGO_SPHERE_VS_CONVEX_POLYHEDRON, batch([
        (SPH_A, BOX_A, (0.1, 0.1, 0.1), I, (0, 0, 0), I),           # centre inside the box (SAT)
        (SPH_A, BOX_A, (0, 0.9, 0), I, (0, 0, 0), I),               # touching the top face (GJK)
        (SPH_A, BOX_A, (1.2, 0.7, 0.9), I, (0, 0, 0), I),           # near a corner
        (SPH_A, BOX_A, (0, 2.0, 0), I, (0, 0, 0), tilt),            # separated
        (SPH_B, HULL, (0.2, 0.1, 0), I, (0, 0, 0), tilt),           # deep in the hull
        (SPH_B, HULL, (0, 1.45, 0), I, (0, 0, 0), I),               # shallow on the hull
        (BOX_A, SPH_A, (0, 0, 0), z45, (0.3, 0.7, 0.1), I),         # box first
        (SPH_A, HULL_S, (0, 0.9, 0.1), I, (0, 0, 0), I),            # scaled hull
    ], cache=True), 16))
    cases.append(("capsule_poly", A.ALGO_CAPSULE_VS_CONVEX_POLYHEDRON, batch([
        (CAP_A, BOX_A, (0, 0.75, 0), z90, (0, 0, 0), I),            # lying on the top face (2 contacts)
        (CAP_A, BOX_A, (0, 0.2, 0), I, (0, 0, 0), I),               # deep, standing
        (CAP_A, BOX_A, (0.2, 1.3, 0), I, (0, 0, 0), I),             # standing on its end
        (CAP_A, BOX_A, (1.1, 0.6, 0), x90, (0, 0, 0), I),           # across a box edge
        (CAP_A, BOX_A, (0, 3.0, 0), tilt, (0, 0, 0), I),            # separated
        (CAP_B, HULL, (0, 1.0, 0), z90, (0, 0, 0), I),              # lying on the hull
        (CAP_B, HULL, (0.1, 0.1, 0.1), tilt, (0, 0, 0), I),         # deep in the hull
        (BOX_A, CAP_A, (0, 0, 0), I, (0, 0.78, 0), z90),            # box first
        (CAP_A, HULL_S, (0, 0.7, 0), z90, (0, 0, 0), I),            # scaled hull
    ], cache=True), 16))
    cases.append(("poly_poly", A.ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON, batch([
        (BOX_B, GROUND, (0, 0.99, 0), I, (0, 0, 0), I),             # resting face to face
        (BOX_B, GROUND, (0, 0.98, 0), y45, (0, 0, 0), I),           # resting, turned 45 deg
        (BOX_B, BOX_B, (0, 0.9, 0), qmul(z45, x90), (0, 0, 0), y45),  # edge across edge
        (BOX_A, BOX_B, (0.3, 0.2, 0.1), tilt, (0, 0, 0), I),        # deep, tilted
        (BOX_B, BOX_B, (0, 3.0, 0), I, (0, 0, 0), I),               # separated
        (HULL, GROUND, (0, 1.25, 0), tilt, (0, 0, 0), I),           # hull on the ground
        (HULL_S, BOX_A, (0.1, 0.9, 0), I, (0, 0, 0), I),            # scaled hull on a box
        (HULL, HULL, (0.5, 1.2, 0.1), tilt, (0, 0, 0), z45),        # hull on hull
        (BOX_A, HULL, (0, 1.2, 0), z45, (0, 0, 0), I),              # box first
        (BOX_B, BOX_B, (0.999, 0, 0), I, (0, 0, 0), I),             # side by side, nearly touching
    ], cache=True), 16))
    rep = np.array([1, 0, 1, 0, 1, 0], np.uint8)
    cases.append(("report_off", A.ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON, batch([
        (BOX_B, GROUND, (0, 0.99, 0), I, (0, 0, 0), I),
        (BOX_B, GROUND, (0, 0.99, 0), I, (0, 0, 0), I),
        (BOX_B, BOX_B, (0, 0.9, 0), qmul(z45, x90), (0, 0, 0), y45),
        (BOX_B, BOX_B, (0, 0.9, 0), qmul(z45, x90), (0, 0, 0), y45),
        (HULL, GROUND, (0, 1.25, 0), tilt, (0, 0, 0), I),
        (HULL, GROUND, (0, 1.25, 0), tilt, (0, 0, 0), I),
    ], report=rep, cache=True), 16))
    cases.append(("report_off_gjk", A.ALGO_CAPSULE_VS_CONVEX_POLYHEDRON, batch([
        (CAP_A, BOX_A, (0, 0.75, 0), z90, (0, 0, 0), I),
        (CAP_A, BOX_A, (0, 0.75, 0), z90, (0, 0, 0), I),
        (CAP_A, BOX_A, (0, 0.2, 0), I, (0, 0, 0), I),
        (CAP_A, BOX_A, (0, 0.2, 0), I, (0, 0, 0), I),
    ], report=np.array([1, 0, 1, 0], np.uint8), cache=True), 16))
    cases.append(("max2", A.ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON, batch([
        (BOX_B, GROUND, (0, 0.99, 0), I, (0, 0, 0), I),
        (BOX_B, GROUND, (0, 0.98, 0), y45, (0, 0, 0), I),
    ], cache=True), 2))
    cases.append(("no_cache", A.ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON, batch([
        (BOX_B, GROUND, (0, 0.99, 0), I, (0, 0, 0), I),
        (HULL, GROUND, (0, 1.25, 0), tilt, (0, 0, 0), I),
    ], cache=False), 16))
    return sh, cases


def load_hull():
    with open(os.path.join(HERE, "golden", "hull42.json")) as fh:
        d = json.load(fh)
    return np.array(d["vertices"], np.float32), [list(map(int, f)) for f in d["faces"]]


def grazing_capsule_batch(n=4096, seed=0):
    """Capsules (CAP_A) lying on the top face of a box (BOX_A, half extents
    1 x 0.5 x 0.75) with their axis almost parallel to one of the face's
    edges and crossing that edge's side plane at a grazing angle, so that
    |n . (b - a)| is below the 1e-4 parallel threshold of
    computePlaneSegmentIntersection and clipSegmentWithPlanes
    (mathematics_functions.h:256-326) takes its one-vertex branch; shallow
    (GJK in margin) and deep (SAT) contacts, both shape orders."""
    rng = np.random.default_rng(seed)
    rows = []
    he = (1.0, 0.5, 0.75)
    for k in range(n):
        along_z = k % 2 == 0
        eps = rng.uniform(-4e-5, 4e-5)
        off = rng.uniform(-2e-5, 2e-5)
        depth = rng.uniform(0.01, 0.25) if k % 4 < 2 else rng.uniform(0.31, 0.45)
        y = he[1] + 0.3 - depth
        side = 1.0 if rng.random() < 0.5 else -1.0
        if along_z:
            # axis (local y) -> world z, then a tiny turn about y
            q = qmul(qaxis((0, 1, 0), math.degrees(eps)), qaxis((1, 0, 0), 90.0))
            pos = (side * he[0] + off, y, rng.uniform(-0.1, 0.1))
        else:
            q = qmul(qaxis((0, 1, 0), math.degrees(eps)), qaxis((0, 0, 1), 90.0))
            pos = (rng.uniform(-0.1, 0.1), y, side * he[2] + off)
        spin = qaxis((0, 1, 0), rng.uniform(0, 360))   # about the capsule's own axis
        qc = qmul(q, spin)
        if k % 8 < 4:
            rows.append((CAP_A, BOX_A, pos, qc, (0.0, 0.0, 0.0), I))
        else:
            rows.append((BOX_A, CAP_A, (0.0, 0.0, 0.0), I, pos, qc))
    return batch(rows)
