"""Seeded synthetic workloads for the narrow-phase hot path.

The narrow-phase microbenchmark draws 1,048,576 shape pairs split over seven
algorithm batches (sphere-sphere, sphere-capsule, capsule-capsule, sphere-box,
capsule-box, box-box, convex hull-box).  Sizes, value ranges and the pair
placement rule are those of the reference workload description: relative
orientation uniform, centre offset direction uniform on the sphere with
length U[0.5, 1.5] x (sum of bounding radii), so about half the pairs touch.
All values are drawn with numpy's PCG64 from a recorded seed and stored as
float32, so every engine that consumes them sees identical bytes.
"""
import json
import os

import numpy as np

from . import _abi as A

BATCH_NAMES = ("sphere_sphere", "sphere_capsule", "capsule_capsule", "sphere_box",
               "capsule_box", "box_box", "hull_box")
BATCH_ALGO = {
    "sphere_sphere": A.ALGO_SPHERE_VS_SPHERE,
    "sphere_capsule": A.ALGO_SPHERE_VS_CAPSULE,
    "capsule_capsule": A.ALGO_CAPSULE_VS_CAPSULE,
    "sphere_box": A.ALGO_SPHERE_VS_CONVEX_POLYHEDRON,
    "capsule_box": A.ALGO_CAPSULE_VS_CONVEX_POLYHEDRON,
    "box_box": A.ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON,
    "hull_box": A.ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON,
}
TOTAL_PAIRS = 1_048_576

REPO_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# Reference QuickHull output for icosphere42_points(); written by tests/golden/make_golden.py.
HULL_FILE = os.path.join(REPO_ROOT, "tests", "golden", "hull42.json")


def batch_sizes(total=TOTAL_PAIRS, nb=7):
    """Even split with the remainder given to the first batches (149,796 each + 4 extra)."""
    base, rem = divmod(total, nb)
    return [base + (1 if i < rem else 0) for i in range(nb)]


def random_quaternions(rng, n):
    """Uniform unit quaternions (Shoemake), returned as float32 (x, y, z, w)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                  b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)], axis=1)
    return q.astype(np.float32)


def random_unit_vectors(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def icosphere42_points(seed=7, radius=0.8, noise=0.05):
    """42-vertex once-subdivided icosahedron of the given radius, each vertex
    pushed radially by U[-noise, noise] (relative)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
         (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    pts = [np.array(p, dtype=np.float64) for p in v]
    mid = {}
    for a, b, c in f:
        for i, j in ((a, b), (b, c), (c, a)):
            key = (min(i, j), max(i, j))
            if key not in mid:
                mid[key] = len(pts)
                pts.append((pts[i] + pts[j]) / 2.0)
    p = np.array(pts)
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    rng = np.random.default_rng(seed)
    scale = radius * (1.0 + rng.uniform(-noise, noise, size=len(p)))
    return (p * scale[:, None]).astype(np.float32)


def load_hull():
    """The hull used by the hull-box batch: vertices and polygon faces as
    produced by the reference's QuickHull on icosphere42_points()."""
    with open(HULL_FILE) as fh:
        d = json.load(fh)
    vertices = np.array(d["vertices"], dtype=np.float32).reshape(-1, 3)
    faces = [list(map(int, f)) for f in d["faces"]]
    return vertices, faces


def _bounding_radius(kind, params, hull_radius):
    if kind == A.SHAPE_SPHERE:
        return params[:, 0]
    if kind == A.SHAPE_CAPSULE:
        return params[:, 0] + params[:, 1]
    if kind == A.SHAPE_BOX:
        return np.linalg.norm(params[:, :3], axis=1)
    return np.full(params.shape[0], hull_radius, dtype=np.float64)


def _draw_shapes(rng, kind, n):
    p = np.zeros((n, 4), dtype=np.float32)
    if kind == A.SHAPE_SPHERE:
        p[:, 0] = rng.uniform(0.2, 1.0, n)
    elif kind == A.SHAPE_CAPSULE:
        p[:, 0] = rng.uniform(0.2, 0.5, n)
        p[:, 1] = rng.uniform(0.3, 1.0, n)
    elif kind == A.SHAPE_BOX:
        p[:, :3] = rng.uniform(0.2, 1.0, (n, 3))
    return p


BATCH_KINDS = {
    "sphere_sphere": (A.SHAPE_SPHERE, A.SHAPE_SPHERE),
    "sphere_capsule": (A.SHAPE_SPHERE, A.SHAPE_CAPSULE),
    "capsule_capsule": (A.SHAPE_CAPSULE, A.SHAPE_CAPSULE),
    "sphere_box": (A.SHAPE_SPHERE, A.SHAPE_BOX),
    "capsule_box": (A.SHAPE_CAPSULE, A.SHAPE_BOX),
    "box_box": (A.SHAPE_BOX, A.SHAPE_BOX),
    "hull_box": (A.SHAPE_CONVEX_MESH, A.SHAPE_BOX),
}


class NarrowphaseScene:
    """Shapes + per-batch pair arrays for the narrow-phase microbenchmark.

    shapes: structured array (rp3dg_shape) holding every shape of every batch.
    batches: dict name -> (algorithm, HostPairs) in BATCH_NAMES order.
    Hull shapes reference convex-mesh instance 0 (the caller registers the
    hull returned by load_hull() once, scale (1,1,1))."""

    def __init__(self, shapes, batches, hull_vertices, hull_faces, seed):
        self.shapes = shapes
        self.batches = batches
        self.hull_vertices = hull_vertices
        self.hull_faces = hull_faces
        self.seed = seed

    @property
    def n_pairs(self):
        return sum(p.n for _, p in self.batches.values())


def narrowphase_scene(total_pairs=TOTAL_PAIRS, seed=1234, names=BATCH_NAMES, position_range=10.0,
                      hull=None):
    rng = np.random.default_rng(seed)
    hull_vertices, hull_faces = hull if hull is not None else load_hull()
    hull_radius = float(np.max(np.linalg.norm(hull_vertices.astype(np.float64), axis=1)))
    sizes = batch_sizes(total_pairs, len(BATCH_NAMES))
    all_shapes = []
    batches = {}
    base = 0
    for name, n in zip(BATCH_NAMES, sizes):
        if name not in names:
            continue
        k1, k2 = BATCH_KINDS[name]
        p1, p2 = _draw_shapes(rng, k1, n), _draw_shapes(rng, k2, n)
        sh = np.zeros(2 * n, dtype=A.SHAPE_DTYPE)
        sh["params"][0::2] = p1
        sh["params"][1::2] = p2
        sh["kind"][0::2] = k1
        sh["kind"][1::2] = k2
        sh["mesh"] = -1
        sh["mesh"][0::2] = 0 if k1 == A.SHAPE_CONVEX_MESH else -1
        sh["mesh"][1::2] = 0 if k2 == A.SHAPE_CONVEX_MESH else -1
        r = (_bounding_radius(k1, p1.astype(np.float64), hull_radius)
             + _bounding_radius(k2, p2.astype(np.float64), hull_radius))
        q1, q2 = random_quaternions(rng, n), random_quaternions(rng, n)
        c1 = rng.uniform(-position_range, position_range, (n, 3))
        d = random_unit_vectors(rng, n) * (rng.uniform(0.5, 1.5, n) * r)[:, None]
        pos1 = np.zeros((n, 4), np.float32)
        pos2 = np.zeros((n, 4), np.float32)
        pos1[:, :3] = c1
        pos2[:, :3] = c1 + d
        idx = base + 2 * np.arange(n, dtype=np.int64)
        pairs = A.HostPairs(idx, idx + 1, pos1, q1, pos2, q2)
        batches[name] = (BATCH_ALGO[name], pairs)
        all_shapes.append(sh)
        base += 2 * n
    shapes = np.concatenate(all_shapes) if all_shapes else np.zeros(0, A.SHAPE_DTYPE)
    return NarrowphaseScene(shapes, batches, hull_vertices, hull_faces, seed)


# ---- worlds ----------------------------------------------------------------

class WorldScene:
    """A world description: settings, shape table, bodies, colliders and
    joints (numpy structured arrays with the layouts of include/rp3dg.h)."""

    def __init__(self, settings, shapes, bodies, colliders, name="", joints=None, heightfields=None,
                 convex_meshes=None, concave_meshes=None):
        self.settings, self.shapes, self.bodies, self.colliders, self.name = settings, shapes, bodies, colliders, name
        self.joints = joints
        # height fields: list of (heights (nb_rows, nb_columns) float32, scale);
        # a SHAPE_HEIGHTFIELD shape's mesh field indexes this list
        self.heightfields = heightfields or []
        # convex meshes: list of (vertices (n, 3), polygon faces, scale); a
        # SHAPE_CONVEX_MESH shape's mesh field indexes this list
        self.convex_meshes = convex_meshes or []
        # concave meshes: list of (vertices (n, 3), triangles (m, 3), vertex
        # normals (n, 3) or None, scale); a SHAPE_CONCAVE_MESH shape's mesh
        # field indexes this list
        self.concave_meshes = concave_meshes or []


def box_pile(nx=10, ny=10, nz=10, seed=1, spacing=2.0, base=2.0, jitter=0.1):
    """The plain box pile: nx*ny*nz dynamic boxes (half-extents U[0.25, 0.75],
    density 1, friction 0.3, bounciness 0) on a grid with `spacing` metres
    between centres, the lowest layer at y = base, each centre jittered by
    U[-jitter, jitter] per axis, uniform random orientations; they fall onto a
    static ground box of half-extents 50 x 0.5 x 50 centred at y = 0.  Gravity
    -9.81, default solver iterations, sleeping on.  Body 0 is the ground."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    shapes = np.zeros(n + 1, A.SHAPE_DTYPE)
    shapes["kind"] = A.SHAPE_BOX
    shapes["mesh"] = -1
    shapes["params"][0, :3] = (50.0, 0.5, 50.0)
    shapes["params"][1:, :3] = rng.uniform(0.25, 0.75, size=(n, 3)).astype(np.float32)
    bodies = A.body_descs(n + 1)
    bodies[0]["type"] = A.BODY_STATIC
    iy, ix, iz = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz), indexing="ij")
    centre = np.stack([(ix.ravel() - 0.5 * (nx - 1)) * spacing, base + iy.ravel() * spacing,
                       (iz.ravel() - 0.5 * (nz - 1)) * spacing], axis=1)
    centre = centre + rng.uniform(-jitter, jitter, size=(n, 3))
    bodies["position"][1:] = centre.astype(np.float32)
    bodies["orientation"][1:] = random_quaternions(rng, n)
    colliders = A.collider_descs(n + 1)
    colliders["body"] = np.arange(n + 1)
    colliders["shape"] = np.arange(n + 1)
    colliders["friction"] = np.float32(0.3)
    colliders["bounciness"] = 0.0
    return WorldScene(A.default_world_settings(), shapes, bodies, colliders, f"box pile {n}")


def hull_world(nx=5, ny=3, nz=5, seed=9, spacing=1.8):
    """Convex hulls (the reference QuickHull of icosphere42_points(), at
    scale 0.6 and at the non-uniform scale (0.7, 0.45, 0.55)), boxes, spheres
    and capsules of random sizes on a jittered grid above a static ground box,
    random orientations; collision categories 1 and 2 alternate."""
    rng = np.random.default_rng(seed)
    verts, faces = load_hull()
    n = nx * ny * nz
    kinds = rng.integers(0, 5, size=n)
    shapes = np.zeros(n + 1, A.SHAPE_DTYPE)
    shapes["mesh"] = -1
    shapes[0]["kind"] = A.SHAPE_BOX
    shapes["params"][0, :3] = (20.0, 0.5, 20.0)
    for i, k in enumerate(kinds):
        sh = shapes[i + 1]
        if k <= 1:
            sh["kind"] = A.SHAPE_CONVEX_MESH
            sh["mesh"] = int(k)
        elif k == 2:
            sh["kind"] = A.SHAPE_BOX
            sh["params"][:3] = rng.uniform(0.25, 0.6, 3)
        elif k == 3:
            sh["kind"] = A.SHAPE_SPHERE
            sh["params"][0] = rng.uniform(0.2, 0.5)
        else:
            sh["kind"] = A.SHAPE_CAPSULE
            sh["params"][:2] = (rng.uniform(0.15, 0.3), rng.uniform(0.2, 0.4))
    bodies = A.body_descs(n + 1)
    bodies[0]["type"] = A.BODY_STATIC
    bodies[0]["position"] = (0.0, -0.5, 0.0)
    iy, ix, iz = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz), indexing="ij")
    centre = np.stack([(ix.ravel() - 0.5 * (nx - 1)) * spacing, 1.0 + iy.ravel() * spacing,
                       (iz.ravel() - 0.5 * (nz - 1)) * spacing], axis=1) + rng.uniform(-0.1, 0.1, size=(n, 3))
    bodies["position"][1:] = centre.astype(np.float32)
    bodies["orientation"][1:] = random_quaternions(rng, n)
    colliders = A.collider_descs(n + 1)
    colliders["body"] = np.arange(n + 1)
    colliders["shape"] = np.arange(n + 1)
    colliders["friction"] = np.float32(0.4)
    colliders["bounciness"] = 0.0
    colliders["category"][1:] = (1 + (np.arange(n) % 2)).astype(np.uint16)
    return WorldScene(A.default_world_settings(), shapes, bodies, colliders, f"hulls {n}",
                      convex_meshes=[(verts, faces, (0.6, 0.6, 0.6)), (verts, faces, (0.7, 0.45, 0.55))])


def world_rays(n, lo, hi, seed=0, down=0.5, max_fraction=1.0, masks=(0xFFFF,)):
    """n rays (A.RAY_DTYPE) for a scene inside the box [lo, hi]: a `down`
    share cast from above the box straight through it with a small random
    tilt, the others between two uniform points of the box grown by a tenth
    of its size; ray k takes category mask masks[k % len(masks)]."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    size = hi - lo
    r = A.rays(n)
    nd = int(n * down)
    p = rng.uniform(lo, hi, size=(nd, 3))
    top = np.array([0.0, hi[1] + 0.5 * size[1] + 1.0, 0.0])
    a = p.copy()
    a[:, 1] = top[1]
    b = p + rng.uniform(-0.05, 0.05, size=(nd, 3)) * size
    b[:, 1] = lo[1] - 0.5 * size[1] - 1.0
    grow = 0.1 * size
    a2 = rng.uniform(lo - grow, hi + grow, size=(n - nd, 3))
    b2 = rng.uniform(lo - grow, hi + grow, size=(n - nd, 3))
    r["point1"] = np.concatenate([a, a2]).astype(np.float32)
    r["point2"] = np.concatenate([b, b2]).astype(np.float32)
    r["max_fraction"] = np.float32(max_fraction)
    r["category_mask"] = np.asarray(masks, np.uint32)[np.arange(n) % len(masks)]
    return r


def terrain_rays(sc, n, seed=41):
    """Rays over the large world: half cast from 5 m above the highest body
    straight down (a random tilt of up to 2% of the footprint), half between
    two uniform points of the world's box (which walk the height field's
    grid when they reach the terrain)."""
    p = sc.bodies["position"][1:]
    half = 0.5 * (np.array(sc.heightfields[0][0].shape[::-1]) - 1)   # (x, z) half-extents of the field
    lo = np.array([-half[0], -4.0, -half[1]])
    hi = np.array([half[0], float(p[:, 1].max()) + 5.0, half[1]])
    rng = np.random.default_rng(seed)
    r = A.rays(n)
    nd = n // 2
    a = rng.uniform(lo, hi, size=(nd, 3))
    a[:, 1] = hi[1]
    b = a + rng.uniform(-0.02, 0.02, size=(nd, 3)) * (hi - lo)
    b[:, 1] = lo[1]
    a2 = rng.uniform(lo, hi, size=(n - nd, 3))
    b2 = rng.uniform(lo, hi, size=(n - nd, 3))
    r["point1"] = np.concatenate([a, a2]).astype(np.float32)
    r["point2"] = np.concatenate([b, b2]).astype(np.float32)
    return r


def mixed_world(nx=5, ny=4, nz=5, seed=2, spacing=1.6, variety=True):
    """Boxes, spheres and capsules of random sizes on a jittered grid above a
    static ground; with `variety`, random frictions and bounciness, dampings,
    lock factors, a few kinematic and gravity-free bodies, initial velocities,
    one body that may not sleep, and collision filters (categories 1, 2, 4;
    every third collider ignores category 2)."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    kinds = rng.integers(0, 3, size=n)
    shapes = np.zeros(n + 1, A.SHAPE_DTYPE)
    shapes["mesh"] = -1
    shapes[0]["kind"] = A.SHAPE_BOX
    shapes["params"][0, :3] = (25.0, 0.25, 25.0)
    for i, k in enumerate(kinds):
        s = shapes[i + 1]
        if k == 0:
            s["kind"] = A.SHAPE_BOX
            s["params"][:3] = rng.uniform(0.25, 0.6, 3)
        elif k == 1:
            s["kind"] = A.SHAPE_SPHERE
            s["params"][0] = rng.uniform(0.2, 0.5)
        else:
            s["kind"] = A.SHAPE_CAPSULE
            s["params"][:2] = (rng.uniform(0.15, 0.3), rng.uniform(0.2, 0.4))
    bodies = A.body_descs(n + 1)
    bodies[0]["type"] = A.BODY_STATIC
    bodies[0]["position"] = (0.0, -0.25, 0.0)
    iy, ix, iz = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz), indexing="ij")
    centre = np.stack([(ix.ravel() - 0.5 * (nx - 1)) * spacing, 1.0 + iy.ravel() * spacing,
                       (iz.ravel() - 0.5 * (nz - 1)) * spacing], axis=1) + rng.uniform(-0.1, 0.1, size=(n, 3))
    bodies["position"][1:] = centre.astype(np.float32)
    bodies["orientation"][1:] = random_quaternions(rng, n)
    colliders = A.collider_descs(n + 1)
    colliders["body"] = np.arange(n + 1)
    colliders["shape"] = np.arange(n + 1)
    colliders["friction"] = np.float32(0.3)
    colliders["bounciness"] = 0.0
    if variety:
        colliders["friction"][1:] = rng.uniform(0.1, 1.0, n).astype(np.float32)
        colliders["bounciness"][1:] = rng.uniform(0.0, 0.6, n).astype(np.float32)
        colliders["friction"][0] = np.float32(0.6)
        for i in range(1, n + 1):
            k = (i - 1) % 23
            b = bodies[i]
            if k == 3:
                b["linear_damping"] = rng.uniform(0.0, 0.5)
            elif k == 4:
                b["angular_damping"] = rng.uniform(0.0, 0.5)
            elif k == 5:
                b["linear_lock"] = (1.0, 0.0, 1.0)
            elif k == 6:
                b["angular_lock"] = (0.0, 1.0, 0.0)
            elif k == 7:
                b["gravity_enabled"] = 0
            elif k == 8:
                b["linear_velocity"] = rng.uniform(-2, 2, 3) * np.array([1, 0.5, 1]) - np.array([0, 1, 0])
            elif k == 9:
                b["angular_velocity"] = rng.uniform(-3, 3, 3)
            elif k == 10:
                b["type"] = A.BODY_KINEMATIC
                b["linear_velocity"] = (rng.uniform(-0.5, 0.5), 0.0, rng.uniform(-0.5, 0.5))
            elif k == 11:
                b["allowed_to_sleep"] = 0
        c = np.arange(n)
        colliders["category"][1:] = (1 << (c % 3)).astype(np.uint16)
        colliders["mask"][1:] = np.where(c % 3 == 0, 0xFFFF & ~2, 0xFFFF).astype(np.uint16)
    return WorldScene(A.default_world_settings(), shapes, bodies, colliders, f"mixed {n}")


def merge_shapes(scenes_):
    """One shape table for several world scenes: the scenes' tables
    concatenated, each scene's collider shape indices shifted (returns the
    table and new scenes; the inputs are not modified)."""
    tables, out, base = [], [], 0
    for s in scenes_:
        c = s.colliders.copy()
        c["shape"] += base
        out.append(WorldScene(s.settings, s.shapes, s.bodies, c, s.name, getattr(s, "joints", None),
                              getattr(s, "heightfields", None), getattr(s, "convex_meshes", None),
                              getattr(s, "concave_meshes", None)))
        tables.append(s.shapes)
        base += len(s.shapes)
    return np.concatenate(tables), out


def many_worlds(n_worlds=4096, seed=7, min_bodies=20, max_bodies=200, spacing=1.2, merge=True, ragdolls=(1, 4),
                limits=True):
    """The many-worlds batch: n_worlds independent worlds with
    U[min_bodies, max_bodies] dynamic bodies each (half boxes with half-extents
    U[0.2, 1], half spheres with radius U[0.2, 1]) stacked on a jittered
    square grid above a static ground box, random orientations, and
    U[ragdolls] ragdolls (ragdoll_world's 15-capsule skeleton, 10
    ball-and-socket + 4 hinge joints, 60-degree cones and +-60-degree hinge
    limits with `limits`) above the stack.
    Returns (shape table, list of WorldScene) with merge, else the scenes with
    their own shape tables."""
    rng = np.random.default_rng(seed)
    scenes_ = []
    for k in range(n_worlds):
        n = int(rng.integers(min_bodies, max_bodies + 1))
        shapes = np.zeros(n + 1, A.SHAPE_DTYPE)
        shapes["mesh"] = -1
        shapes[0]["kind"] = A.SHAPE_BOX
        shapes["params"][0, :3] = (25.0, 0.5, 25.0)
        kinds = rng.integers(0, 2, n)
        shapes["kind"][1:] = np.where(kinds == 0, A.SHAPE_BOX, A.SHAPE_SPHERE)
        shapes["params"][1:, :3] = rng.uniform(0.2, 1.0, size=(n, 3)).astype(np.float32)
        side = int(np.ceil(np.sqrt(n / 4.0)))
        idx = np.arange(n)
        gx, gz, gy = idx % side, (idx // side) % side, idx // (side * side)
        centre = np.stack([(gx - 0.5 * (side - 1)) * 2.2 * spacing, 1.5 + gy * 2.2 * spacing,
                           (gz - 0.5 * (side - 1)) * 2.2 * spacing], axis=1) + rng.uniform(-0.1, 0.1, (n, 3))
        nr = int(rng.integers(ragdolls[0], ragdolls[1] + 1)) if ragdolls else 0
        nparts = len(RAGDOLL_PARTS)
        shapes = np.concatenate([shapes, np.zeros(nr * nparts, A.SHAPE_DTYPE)])
        shapes["mesh"][n + 1:] = -1
        bodies = A.body_descs(n + 1 + nr * nparts)
        bodies[0]["type"] = A.BODY_STATIC
        bodies["position"][1:n + 1] = centre.astype(np.float32)
        bodies["orientation"][1:n + 1] = random_quaternions(rng, n)
        top = float(centre[:, 1].max()) + 2.5
        joints = []
        b = n + 1
        for r in range(nr):
            base = np.array([(r - 0.5 * (nr - 1)) * 3.0, top, 0.0]) + rng.uniform(-0.2, 0.2, 3)
            params, centres, q, js = _ragdoll(rng, b, base, limits)
            shapes["kind"][b:b + nparts] = A.SHAPE_CAPSULE
            shapes["params"][b:b + nparts, :2] = params
            bodies["position"][b:b + nparts] = centres.astype(np.float32)
            bodies["orientation"][b:b + nparts] = np.asarray(q, dtype=np.float32)
            joints += js
            b += nparts
        nt = len(bodies)
        colliders = A.collider_descs(nt)
        colliders["body"] = np.arange(nt)
        colliders["shape"] = np.arange(nt)
        colliders["friction"] = np.float32(0.3)
        colliders["bounciness"] = 0.0
        scenes_.append(WorldScene(A.default_world_settings(), shapes, bodies, colliders,
                                  f"world {k} ({n} bodies, {nr} ragdolls)",
                                  np.array(joints, dtype=A.JOINT_DESC_DTYPE) if joints else None))
    return merge_shapes(scenes_) if merge else scenes_


# 15-part skeleton: (name, parent index, offset of the part's centre from the
# parent's centre in the ragdoll frame, joint: "ball" or "hinge")
RAGDOLL_PARTS = (
    ("pelvis", -1, (0.0, 0.0, 0.0), None),
    ("spine", 0, (0.0, 0.35, 0.0), "ball"),
    ("chest", 1, (0.0, 0.35, 0.0), "ball"),
    ("neck", 2, (0.0, 0.3, 0.0), "ball"),
    ("head", 3, (0.0, 0.25, 0.0), "ball"),
    ("l_upper_arm", 2, (0.35, 0.1, 0.0), "ball"),
    ("l_forearm", 5, (0.4, 0.0, 0.0), "hinge"),
    ("l_hand", 6, (0.3, 0.0, 0.0), "ball"),
    ("r_upper_arm", 2, (-0.35, 0.1, 0.0), "ball"),
    ("r_forearm", 8, (-0.4, 0.0, 0.0), "hinge"),
    ("r_hand", 9, (-0.3, 0.0, 0.0), "ball"),
    ("l_thigh", 0, (0.15, -0.45, 0.0), "ball"),
    ("l_shin", 11, (0.0, -0.5, 0.0), "hinge"),
    ("r_thigh", 0, (-0.15, -0.45, 0.0), "ball"),
    ("r_shin", 13, (0.0, -0.5, 0.0), "hinge"),
)


def _rotate(q, v):
    """Rotate vectors v (n, 3) by the unit quaternion q (x, y, z, w), float64."""
    x, y, z, w = q
    u = np.array([x, y, z])
    v = np.asarray(v, dtype=np.float64)
    return v + 2.0 * np.cross(u, np.cross(u, v) + w * v)


def _ragdoll(rng, first, base, limits):
    """One ragdoll whose first body index is `first`, centred at `base` with a
    random orientation: (capsule params (15, 2), centres (15, 3), orientation,
    joint records)."""
    nparts = len(RAGDOLL_PARTS)
    q = random_quaternions(rng, 1)[0].astype(np.float64)
    centres = np.zeros((nparts, 3))
    for i, (_, parent, off, _) in enumerate(RAGDOLL_PARTS):
        centres[i] = (centres[parent] if parent >= 0 else 0.0) + np.array(off)
    world_c = _rotate(q, centres) + base
    params = np.stack([rng.uniform(0.08, 0.15, nparts), rng.uniform(0.1, 0.3, nparts)], axis=1)
    joints = []
    for i, (_, parent, _, kind) in enumerate(RAGDOLL_PARTS):
        if parent < 0:
            continue
        j = A.joint_descs(1)[0]
        j["type"] = A.JOINT_HINGE if kind == "hinge" else A.JOINT_BALL_AND_SOCKET
        j["body1"], j["body2"] = first + parent, first + i
        j["anchor"] = (0.5 * (world_c[parent] + world_c[i])).astype(np.float32)
        j["axis"] = _rotate(q, np.array([[0.0, 0.0, 1.0]]))[0].astype(np.float32)
        j["collision_enabled"] = 0
        if limits:
            if kind == "hinge":
                j["limit_enabled"] = 1
                j["min_angle"] = np.float32(-np.pi / 3)
                j["max_angle"] = np.float32(np.pi / 3)
            else:
                j["cone_limit_enabled"] = 1
                j["cone_half_angle"] = np.float32(np.pi / 3)
        joints.append(j)
    return params, world_c, q, joints


def ragdoll_world(n_ragdolls=2, seed=21, limits=True, boxes=0):
    """Ragdolls (15 capsules each: radius U[0.08, 0.15], half-height
    U[0.1, 0.3]; 10 ball-and-socket and 4 hinge joints in a tree, the bodies
    a joint connects not colliding with each other, as in the reference
    testbed's ragdoll scene) dropped with random orientations onto a static
    ground box, optionally with a few boxes.  With limits, the ball-and-socket
    joints have a 60-degree cone and the hinges (elbows, knees) +-60 degrees
    (tolerance-level parity: the reference computes these angles with
    acos / atan2)."""
    rng = np.random.default_rng(seed)
    nparts = len(RAGDOLL_PARTS)
    n = 1 + n_ragdolls * nparts + boxes
    shapes = np.zeros(n, A.SHAPE_DTYPE)
    shapes["mesh"] = -1
    shapes[0]["kind"] = A.SHAPE_BOX
    shapes["params"][0, :3] = (25.0, 0.5, 25.0)
    bodies = A.body_descs(n)
    bodies[0]["type"] = A.BODY_STATIC
    joints = []
    b = 1
    for r in range(n_ragdolls):
        base = np.array([(r % 4) * 3.0 - 4.5, 2.5 + 1.0 * (r // 4), (r // 4) * 2.0 - 2.0]) + rng.uniform(-0.2, 0.2, 3)
        params, centres, q, js = _ragdoll(rng, b, base, limits)
        shapes["kind"][b:b + nparts] = A.SHAPE_CAPSULE
        shapes["params"][b:b + nparts, :2] = params
        bodies["position"][b:b + nparts] = centres.astype(np.float32)
        bodies["orientation"][b:b + nparts] = np.asarray(q, dtype=np.float32)
        joints += js
        b += nparts
    for k in range(boxes):
        shapes[b]["kind"] = A.SHAPE_BOX
        shapes[b]["params"][:3] = rng.uniform(0.2, 0.5, 3)
        bodies[b]["position"] = (rng.uniform(-4, 4), 0.8 + 0.6 * k, rng.uniform(-3, 3))
        bodies[b]["orientation"] = random_quaternions(rng, 1)[0]
        b += 1
    colliders = A.collider_descs(n)
    colliders["body"] = np.arange(n)
    colliders["shape"] = np.arange(n)
    colliders["friction"] = np.float32(0.3)
    colliders["bounciness"] = 0.0
    return WorldScene(A.default_world_settings(), shapes, bodies, colliders,
                      f"ragdolls {n_ragdolls}", np.array(joints, dtype=A.JOINT_DESC_DTYPE))


def _yaw_quaternion(angle):
    return np.array([0.0, np.sin(0.5 * angle), 0.0, np.cos(0.5 * angle)])


def mechanism_world(n_mechanisms=1, seed=31, spacing=20.0, speeds=(-2.0, 2.0)):
    """Copies of the reference testbed's joints scene (testbed/scenes/joints/
    JointsScene.cpp) on one static floor, each turned by a random yaw about
    its centre: a chain of 7 unit boxes hanging from a static box by 6
    ball-and-socket joints; a dynamic box (1.5 x 4 x 1.5) on a slider joint
    over a static box (2 x 4 x 2), translation limits +-1.7 and a motor
    (random speed in `speeds`, max force 10000); a propeller box (10 x 1 x 1)
    on a motorised hinge (-PI / 2 rad/s, max torque 60) above the sliding box;
    and two boxes (1.5 cubed) welded to the propeller's ends by fixed joints.
    The bodies a joint connects do not collide; boxes have bounciness 0.4,
    chain boxes angular damping 0.2.  The mechanisms sit on a square grid
    `spacing` metres apart on a floor 0.5 m thick."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(np.sqrt(n_mechanisms)))
    half_floor = 0.5 * side * spacing + 5.0
    # (half extents, centre, static) of one mechanism's bodies, in its frame
    parts = [((0.5, 0.5, 0.5), (0.0, 15.0 - 1.5 * i, 5.0), i == 0) for i in range(7)]
    parts += [((1.0, 2.0, 1.0), (0.0, 2.1, 0.0), True), ((0.75, 2.0, 0.75), (0.0, 4.2, 0.0), False),
              ((5.0, 0.5, 0.5), (0.0, 7.0, 0.0), False),
              ((0.75, 0.75, 0.75), (5.0, 7.0, 0.0), False), ((0.75, 0.75, 0.75), (-5.0, 7.0, 0.0), False)]
    per = len(parts)
    n = 1 + n_mechanisms * per
    shapes = np.zeros(n, A.SHAPE_DTYPE)
    shapes["mesh"] = -1
    shapes["kind"] = A.SHAPE_BOX
    shapes["params"][0, :3] = (half_floor, 0.25, half_floor)
    bodies = A.body_descs(n)
    bodies[0]["type"] = A.BODY_STATIC
    colliders = A.collider_descs(n)
    colliders["body"] = np.arange(n)
    colliders["shape"] = np.arange(n)
    colliders["bounciness"] = np.float32(0.4)
    colliders[0]["bounciness"] = np.float32(0.3)
    joints = []
    for m in range(n_mechanisms):
        b = 1 + m * per
        origin = np.array([(m % side - 0.5 * (side - 1)) * spacing, 0.0, (m // side - 0.5 * (side - 1)) * spacing])
        q = _yaw_quaternion(rng.uniform(0.0, 2.0 * np.pi))
        centres = _rotate(q, np.array([c for _, c, _ in parts])) + origin
        c32 = centres.astype(np.float32)
        for k, (he, _, static) in enumerate(parts):
            shapes["params"][b + k, :3] = he
            bodies[b + k]["position"] = c32[k]
            bodies[b + k]["orientation"] = q.astype(np.float32)
            if static:
                bodies[b + k]["type"] = A.BODY_STATIC
            if k < 7:
                bodies[b + k]["angular_damping"] = np.float32(0.2)

        def joint(kind, i1, i2, anchor, axis=None):
            j = A.joint_descs(1)[0]
            j["type"] = kind
            j["body1"], j["body2"] = b + i1, b + i2
            j["anchor"] = np.asarray(anchor, dtype=np.float32)
            if axis is not None:
                j["axis"] = np.asarray(axis, dtype=np.float32)
            return j
        for i in range(6):
            j = joint(A.JOINT_BALL_AND_SOCKET, i, i + 1, 0.5 * (c32[i].astype(np.float64) + c32[i + 1]))
            joints.append(j)
        j = joint(A.JOINT_SLIDER, 7, 8, np.float32(0.5) * (c32[8] + c32[7]), c32[8] - c32[7])
        j["collision_enabled"] = 0
        j["limit_enabled"] = 1
        j["min_angle"], j["max_angle"] = np.float32(-1.7), np.float32(1.7)
        j["motor_enabled"] = 1
        j["motor_speed"] = np.float32(rng.uniform(*speeds))
        j["max_motor_torque"] = np.float32(10000.0)
        joints.append(j)
        j = joint(A.JOINT_HINGE, 9, 8, 0.5 * (c32[8].astype(np.float64) + c32[9]), _rotate(q, [[0.0, 1.0, 0.0]])[0])
        j["collision_enabled"] = 0
        j["motor_enabled"] = 1
        j["motor_speed"] = -np.float32(0.5) * np.float32(3.141592653589)
        j["max_motor_torque"] = np.float32(60.0)
        joints.append(j)
        for k in (10, 11):
            j = joint(A.JOINT_FIXED, k, 9, c32[k])
            j["collision_enabled"] = 0
            joints.append(j)
    return WorldScene(A.default_world_settings(), shapes, bodies, colliders, f"mechanisms {n_mechanisms}",
                      np.array(joints, dtype=A.JOINT_DESC_DTYPE))


def mechanism_motor_speeds(n_mechanisms, step, dt=1.0 / 60.0):
    """The slider motor speeds before update `step` (0-based) of
    mechanism_world: (joint index, speed) pairs, speed 2 cos(1.5 t + m) m/s at
    elapsed time t = step * dt for mechanism m, as the testbed's joints scene
    drives its slider (JointsScene::updatePhysics)."""
    t = step * float(dt)
    return [(10 * m + 6, np.float32(2.0 * np.cos(1.5 * t + m))) for m in range(n_mechanisms)]


def sine_heights(cols, rows, seed=3, n_waves=8, amplitude=2.0, k_range=(0.05, 0.5), cell=1.0):
    """A height grid (rows, cols) of `n_waves` sines with random directions,
    wave numbers |k| in k_range (rad per metre) and phases, whose amplitudes
    sum to `amplitude` metres; computed in float64, stored as float32."""
    rng = np.random.default_rng(seed)
    x = np.arange(cols) * cell
    z = np.arange(rows) * cell
    X, Z = np.meshgrid(x, z)
    h = np.zeros((rows, cols))
    for _ in range(n_waves):
        k = rng.uniform(*k_range)
        th = rng.uniform(0.0, 2.0 * np.pi)
        ph = rng.uniform(0.0, 2.0 * np.pi)
        h += (amplitude / n_waves) * np.sin(k * (np.cos(th) * X + np.sin(th) * Z) + ph)
    return h.astype(np.float32)


def heightfield_world(n_bodies=1000, cols=64, rows=64, cell=1.0, seed=5, spacing=1.5, amplitude=2.0,
                      sleeping=True, y_scale=1.0, terrain_position=(0.0, 0.0, 0.0), terrain_orientation=None):
    """Bodies over a static height-field terrain: n_bodies dynamic bodies,
    40% boxes (half-extents U[0.2, 0.6]), 30% spheres (radius U[0.2, 0.5]),
    30% capsules (radius 0.2, half-height 0.3), on a jittered 3-D lattice with
    `spacing` metres between centres above a cols x rows height field of
    `cell`-metre cells whose heights are sine_heights (total amplitude
    `amplitude`).  Body 0 is the terrain (a static body at the origin whose
    collider is the height field, scaled by (cell, y_scale, cell), placed at
    terrain_position with terrain_orientation (x, y, z, w), identity by
    default).  Density 1, friction 0.3, gravity -9.81."""
    rng = np.random.default_rng(seed)
    heights = sine_heights(cols, rows, seed=seed + 1000, amplitude=amplitude, cell=cell)
    n = n_bodies
    shapes = np.zeros(n + 1, A.SHAPE_DTYPE)
    shapes["mesh"] = -1
    shapes[0]["kind"] = A.SHAPE_HEIGHTFIELD
    shapes[0]["mesh"] = 0
    u = rng.uniform(size=n)
    kinds = np.where(u < 0.4, A.SHAPE_BOX, np.where(u < 0.7, A.SHAPE_SPHERE, A.SHAPE_CAPSULE))
    shapes["kind"][1:] = kinds
    box = kinds == A.SHAPE_BOX
    sph = kinds == A.SHAPE_SPHERE
    cap = kinds == A.SHAPE_CAPSULE
    p = shapes["params"][1:]
    p[box, :3] = rng.uniform(0.2, 0.6, size=(int(box.sum()), 3))
    p[sph, 0] = rng.uniform(0.2, 0.5, size=int(sph.sum()))
    p[cap, 0] = 0.2
    p[cap, 1] = 0.3
    shapes["params"][1:] = p
    bodies = A.body_descs(n + 1)
    bodies[0]["type"] = A.BODY_STATIC
    bodies[0]["position"] = terrain_position
    if terrain_orientation is not None:
        bodies[0]["orientation"] = terrain_orientation
    # lattice over the terrain, 1 m inside its border, layers upwards
    width, length = (cols - 1) * cell, (rows - 1) * cell
    nx = max(1, int((width - 2.0) // spacing) + 1)
    nz = max(1, int((length - 2.0) // spacing) + 1)
    per_layer = nx * nz
    idx = np.arange(n)
    iy, rem = idx // per_layer, idx % per_layer
    ix, iz = rem % nx, rem // nx
    top = float(heights.max() - heights.min()) * 0.5 * y_scale + float(terrain_position[1])
    centre = np.stack([(ix - 0.5 * (nx - 1)) * spacing, top + 1.5 + iy * spacing,
                       (iz - 0.5 * (nz - 1)) * spacing], axis=1) + rng.uniform(-0.1, 0.1, size=(n, 3))
    bodies["position"][1:] = centre.astype(np.float32)
    bodies["orientation"][1:] = random_quaternions(rng, n)
    colliders = A.collider_descs(n + 1)
    colliders["body"] = np.arange(n + 1)
    colliders["shape"] = np.arange(n + 1)
    colliders["friction"] = np.float32(0.3)
    colliders["bounciness"] = 0.0
    settings = A.default_world_settings()
    settings["sleeping_enabled"] = 1 if sleeping else 0
    return WorldScene(settings, shapes, bodies, colliders, f"heightfield {cols}x{rows} + {n}",
                      heightfields=[(heights, (cell, y_scale, cell))])


def with_triggers(scene, every=6, zones=((0.0, 2.0, 0.0, 2.5, 0.6, 2.5), (-3.0, 4.5, 1.0, 1.5, 1.5, 1.5))):
    """A copy of `scene` with trigger colliders (Collider::setIsTrigger): every
    `every`-th dynamic body's collider becomes a trigger (the body keeps its
    mass, falls through everything and reports overlaps), and static trigger
    boxes are added as sensor zones, one per (x, y, z, half-extent x, y, z)."""
    shapes = np.concatenate([scene.shapes, np.zeros(len(zones), A.SHAPE_DTYPE)])
    bodies = np.concatenate([scene.bodies, A.body_descs(len(zones))])
    colliders = np.concatenate([scene.colliders, A.collider_descs(len(zones))])
    dyn = np.flatnonzero(scene.bodies["type"] == A.BODY_DYNAMIC)
    for b in dyn[::every]:
        colliders["flags"][np.flatnonzero(scene.colliders["body"] == b)] |= A.COLLIDER_TRIGGER
    ns, nb, nc = len(scene.shapes), len(scene.bodies), len(scene.colliders)
    for k, (x, y, z, hx, hy, hz) in enumerate(zones):
        shapes["kind"][ns + k] = A.SHAPE_BOX
        shapes["mesh"][ns + k] = -1
        shapes["params"][ns + k, :3] = (hx, hy, hz)
        bodies["type"][nb + k] = A.BODY_STATIC
        bodies["position"][nb + k] = (x, y, z)
        colliders["body"][nc + k] = nb + k
        colliders["shape"][nc + k] = ns + k
        colliders["flags"][nc + k] = A.COLLIDER_TRIGGER
    return WorldScene(scene.settings, shapes, bodies, colliders, scene.name + " with triggers",
                      getattr(scene, "joints", None), getattr(scene, "heightfields", None),
                      getattr(scene, "convex_meshes", None), getattr(scene, "concave_meshes", None))


def terrain_mesh(cols=24, rows=24, cell=1.0, seed=61, amplitude=2.0, jitter=0.2):
    """A triangle-mesh terrain: a cols x rows grid of vertices at
    sine_heights, x and z jittered by up to `jitter` cells, two triangles per
    cell wound upwards (the height field's (p1, p2, p3), (p3, p2, p4) order),
    the diagonal alternating from cell to cell; plus what
    TriangleMesh::init must clean up: an unused vertex in the middle of the
    array and two degenerate triangles (a repeated index, a zero-length
    edge).  Returns (vertices (n, 3) float32, triangles (m, 3) uint32)."""
    rng = np.random.default_rng(seed)
    h = sine_heights(cols, rows, seed=seed + 1000, amplitude=amplitude, cell=cell)
    I, J = np.meshgrid(np.arange(cols), np.arange(rows), indexing="ij")
    x = (I - 0.5 * (cols - 1)) * cell + rng.uniform(-jitter, jitter, I.shape) * cell
    z = (J - 0.5 * (rows - 1)) * cell + rng.uniform(-jitter, jitter, I.shape) * cell
    y = h.T   # h is (rows, cols): row j along z, column i along x
    verts = np.stack([x, y, z], axis=-1).reshape(-1, 3).astype(np.float32)
    vid = lambda i, j: i * rows + j
    tris = []
    for i in range(cols - 1):
        for j in range(rows - 1):
            p1, p2, p3, p4 = vid(i, j), vid(i, j + 1), vid(i + 1, j), vid(i + 1, j + 1)
            if (i + j) % 2 == 0:
                tris += [(p1, p2, p3), (p3, p2, p4)]
            else:
                tris += [(p1, p2, p4), (p1, p4, p3)]
    # an unused vertex in the middle, shifting the later indices
    mid = len(verts) // 2
    verts = np.concatenate([verts[:mid], np.array([[0.0, 50.0, 0.0]], np.float32), verts[mid:]])
    tris = [tuple(v + (v >= mid) for v in t) for t in tris]
    tris.insert(len(tris) // 3, (tris[0][0], tris[0][0], tris[0][1]))   # zero-length edge
    tris.append((tris[5][1], tris[5][2], tris[5][2]))
    return verts, np.array(tris, np.uint32)


def concave_mesh_world(n_bodies=300, cols=24, rows=24, cell=1.0, seed=61, spacing=1.5, amplitude=2.0, hulls=True,
                       scale=(1.0, 1.0, 1.0), normals=False, terrain_orientation=None, sleeping=True):
    """Bodies over a static concave-mesh terrain (terrain_mesh, scaled by
    `scale`; vertex normals computed by TriangleMesh::init, or given as the
    normalised up vector when `normals`): n_bodies dynamic bodies, boxes,
    spheres and capsules (and convex hulls when `hulls`) on a jittered
    lattice above the terrain.  Body 0 is the terrain, static at the origin
    with terrain_orientation (x, y, z, w), identity by default."""
    rng = np.random.default_rng(seed)
    verts, tris = terrain_mesh(cols, rows, cell, seed, amplitude)
    vn = None
    if normals:
        vn = np.tile(np.array([[0.0, 1.0, 0.0]], np.float32), (len(verts), 1))
        vn[:, 0] = rng.uniform(-0.2, 0.2, len(verts))
        vn /= np.linalg.norm(vn, axis=1, keepdims=True)
        vn = vn.astype(np.float32)
    n = n_bodies
    shapes = np.zeros(n + 1, A.SHAPE_DTYPE)
    shapes["mesh"] = -1
    shapes[0]["kind"] = A.SHAPE_CONCAVE_MESH
    shapes[0]["mesh"] = 0
    kinds = rng.integers(0, 5 if hulls else 3, size=n)
    convex = []
    if hulls:
        hv, hf = load_hull()
        convex = [(hv, hf, (0.5, 0.5, 0.5)), (hv, hf, (0.6, 0.4, 0.5))]
    for i, k in enumerate(kinds):
        sh = shapes[i + 1]
        if k == 0:
            sh["kind"] = A.SHAPE_BOX
            sh["params"][:3] = rng.uniform(0.2, 0.5, 3)
        elif k == 1:
            sh["kind"] = A.SHAPE_SPHERE
            sh["params"][0] = rng.uniform(0.2, 0.45)
        elif k == 2:
            sh["kind"] = A.SHAPE_CAPSULE
            sh["params"][:2] = (rng.uniform(0.15, 0.25), rng.uniform(0.2, 0.35))
        else:
            sh["kind"] = A.SHAPE_CONVEX_MESH
            sh["mesh"] = int(k - 3)
    bodies = A.body_descs(n + 1)
    bodies[0]["type"] = A.BODY_STATIC
    if terrain_orientation is not None:
        bodies[0]["orientation"] = terrain_orientation
    width, length = (cols - 1) * cell * scale[0], (rows - 1) * cell * scale[2]
    nx = max(1, int((width - 3.0) // spacing) + 1)
    nz = max(1, int((length - 3.0) // spacing) + 1)
    per_layer = nx * nz
    idx = np.arange(n)
    iy, rem = idx // per_layer, idx % per_layer
    ix, iz = rem % nx, rem // nx
    top = float(verts[:, 1][verts[:, 1] < 40.0].max()) * scale[1]
    centre = np.stack([(ix - 0.5 * (nx - 1)) * spacing, top + 1.5 + iy * spacing,
                       (iz - 0.5 * (nz - 1)) * spacing], axis=1) + rng.uniform(-0.1, 0.1, size=(n, 3))
    bodies["position"][1:] = centre.astype(np.float32)
    bodies["orientation"][1:] = random_quaternions(rng, n)
    colliders = A.collider_descs(n + 1)
    colliders["body"] = np.arange(n + 1)
    colliders["shape"] = np.arange(n + 1)
    colliders["friction"] = np.float32(0.4)
    colliders["bounciness"] = 0.0
    settings = A.default_world_settings()
    settings["sleeping_enabled"] = 1 if sleeping else 0
    return WorldScene(settings, shapes, bodies, colliders, f"concave mesh {cols}x{rows} + {n}",
                      convex_meshes=convex, concave_meshes=[(verts, tris, vn, tuple(map(float, scale)))])
