"""Regenerates the golden fixtures under tests/golden/ from the reference
engine itself (oracle/_ref/librp3d_ref_f32.so, built by `make -C oracle ref`
from the reference's own sources).  Run from the repository root:

    python tests/golden/make_golden.py

Writes:
  hull42.json      the reference QuickHull of the seeded 42-point icosphere
                   (the convex hull used by the hull-box workload)
  np_scene.npz     a small seeded narrow-phase scene (all seven batches) with
                   the reference's per-pair outputs and caches: pass "a" with
                   fresh caches, pass "b" with slightly moved poses and the
                   caches of pass "a" marked valid (temporal-coherence paths)
  np_edge.npz      hand-placed degenerate and boundary cases (coincident
                   centres, centre on a capsule axis, parallel and crossing
                   capsules, resting and edge-crossing boxes, deep and
                   margin-only sphere/capsule vs box and hull, reversed shape
                   order, report_contacts off, a scaled hull, max_contacts 2)
  np_manifold.npz  contact-manifold reduction: per batch of a seeded scene,
                   the reference narrow phase's raw points of selected pairs
                   (every pair with more than 4 points, up to 160, plus
                   colliding pairs with 1-4 points and separated pairs), and
                   the reference's reduceContactPoints +
                   removeDuplicatedContactPointsInManifold result ("red_"
                   arrays and the kept-slot table)

  np_dynamics.npz  one captured step of seeded reference worlds
                   (oracle/ref_world.cpp: boxes, or boxes, spheres and
                   capsules with random materials, dampings, lock factors,
                   forces, kinematic bodies and collision filters, on a
                   static ground): the reference's own inputs and outputs of
                   the dynamics stage (inertia / velocities / contact solver /
                   positions / state: "<case>/in_*", "<case>/out_*",
                   "<case>/params") and of the broad phase (fat AABBs before
                   and after the collider update, moved colliders, the
                   overlapping pairs after the step's broad phase, shapes and
                   filter bits: "<case>/bp_*")

  world.npz        whole world steps of two seeded scenes (tests/worldio.py:
                   a 125-box pile for 240 steps, a mixed world of boxes,
                   spheres and capsules with materials, dampings, locks,
                   kinematic / gravity-free bodies and filters for 200 steps,
                   four ragdolls of ball-and-socket and hinge joints without
                   limits with six boxes for 240 steps)
                   stepped by the reference's PhysicsWorld::update: per step
                   the overlapping-pair ids in array order and the solver's
                   manifolds (counts + 64-bit digests), and the body states
                   at checkpoints, bit for bit

`python tests/golden/make_golden.py manifold` (or `dynamics`, `world`)
rewrites that fixture only.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from reactphysics3d_b200 import _abi as A  # noqa: E402
from reactphysics3d_b200 import scenes  # noqa: E402
import goldenio  # noqa: E402
import reflib  # noqa: E402
import edgecases  # noqa: E402


MANIFOLD_FIELDS = ("is_colliding", "nb_contacts", "normal_depth", "local1", "local2")


def pick(c, idx, max_contacts):
    """The pairs idx of a HostContacts, keeping max_contacts slots."""
    s = A.HostContacts(len(idx), max_contacts)
    s.is_colliding[:] = c.is_colliding[idx]
    s.nb_contacts[:] = c.nb_contacts[idx]
    for f in ("normal_depth", "local1", "local2"):
        getattr(s, f)[...] = getattr(c, f)[:max_contacts, idx]
    return s


def manifold_fixture(ref, verts, faces):
    sc = scenes.narrowphase_scene(total_pairs=7 * 8192, seed=29, hull=(verts, faces))
    d = {}
    rng = np.random.default_rng(30)
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        out, _ = ref.narrowphase(algo, sc.shapes, pairs.slice(0, pairs.n))
        col = out.is_colliding.astype(bool)
        many = np.flatnonzero(col & (out.nb_contacts > 4))[:160]
        few = np.flatnonzero(col & (out.nb_contacts > 0) & (out.nb_contacts <= 4))
        sep = np.flatnonzero(~col)
        few = rng.choice(few, size=min(48, len(few)), replace=False) if len(few) else few
        sep = rng.choice(sep, size=min(8, len(sep)), replace=False) if len(sep) else sep
        idx = np.sort(np.concatenate([many, few, sep]).astype(np.int64))
        mc = max(4, int(out.nb_contacts[idx].max()) if len(idx) else 4)
        raw = pick(out, idx, mc)
        sub = A.HostPairs(pairs.shape1[idx], pairs.shape2[idx], pairs.pos1[idx], pairs.rot1[idx],
                          pairs.pos2[idx], pairs.rot2[idx])
        red = reflib.copy_contacts(raw)
        kept = reflib.reduce_contacts(ref.lib, "ref_reduce_contacts", sub, red)
        d[name + "_pos1"], d[name + "_rot1"] = sub.pos1, sub.rot1
        for f in MANIFOLD_FIELDS:
            d[name + "_" + f] = getattr(raw, f)
            d[name + "_red_" + f] = getattr(red, f)
        d[name + "_kept"] = kept
        print(name, "pairs", len(idx), ">4:", len(many), "max points", mc,
              "de-duplicated:", int(np.sum(np.minimum(raw.nb_contacts, 4) != red.nb_contacts)))
    pairs, raw = synthetic_manifolds(np.random.default_rng(31))
    red = reflib.copy_contacts(raw)
    kept = reflib.reduce_contacts(ref.lib, "ref_reduce_contacts", pairs, red)
    d["synthetic_pos1"], d["synthetic_rot1"] = pairs.pos1, pairs.rot1
    for f in MANIFOLD_FIELDS:
        d["synthetic_" + f] = getattr(raw, f)
        d["synthetic_red_" + f] = getattr(red, f)
    d["synthetic_kept"] = kept
    print("synthetic pairs", pairs.n, "de-duplicated:",
          int(np.sum(np.minimum(raw.nb_contacts, 4) != red.nb_contacts)))
    np.savez_compressed(os.path.join(HERE, "np_manifold.npz"), **d)


def synthetic_manifolds(rng, n=512):
    """Raw manifolds the reduction must handle beyond what a narrow phase
    emits often: 1-16 points, exact and near (< 0.01) duplicates, collinear
    and coincident sets, points on a grid (equal dot products and areas), a
    separated pair that still holds points."""
    mc = A.MAX_CONTACTS
    c = A.HostContacts(n, mc)
    q = rng.normal(size=(n, 4)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    for i in range(n):
        kind = i % 8
        nb = int(rng.integers(1, mc + 1)) if kind != 7 else int(rng.integers(5, mc + 1))
        if kind == 0:
            p = rng.uniform(-1, 1, size=(nb, 3))
        elif kind == 1:       # exact duplicates
            base = rng.uniform(-1, 1, size=(max(1, nb // 2), 3))
            p = base[rng.integers(0, len(base), size=nb)]
        elif kind == 2:       # near duplicates, within and just outside 0.01
            base = rng.uniform(-1, 1, size=(max(1, nb // 3), 3))
            p = base[rng.integers(0, len(base), size=nb)] + rng.normal(scale=0.006, size=(nb, 3))
        elif kind == 3:       # collinear
            t = rng.uniform(-1, 1, size=(nb, 1))
            p = rng.uniform(-1, 1, size=(1, 3)) + t * rng.normal(size=(1, 3))
        elif kind == 4:       # all the same point
            p = np.repeat(rng.uniform(-1, 1, size=(1, 3)), nb, axis=0)
        elif kind == 5:       # a grid in a plane: ties in every comparison
            g = np.array([(x, y, 0.0) for x in range(4) for y in range(4)], np.float64) * 0.25
            p = g[rng.permutation(16)[:nb]]
        elif kind == 6:       # a box-face octagon with the normal along z
            a = np.arange(nb) * (2 * np.pi / nb)
            p = np.stack([np.cos(a), np.sin(a), np.zeros(nb)], 1)
            nrm[i] = (0.0, 0.0, 1.0)
            q[i] = (0.0, 0.0, 0.0, 1.0)
        else:
            p = rng.uniform(-1, 1, size=(nb, 3)) * np.array([1.0, 1.0, 1e-3])
        c.nb_contacts[i] = nb
        c.is_colliding[i] = 0 if i % 61 == 60 else 1
        c.normal_depth[:nb, i, :3] = nrm[i]
        c.normal_depth[:nb, i, 3] = rng.uniform(0.001, 0.2, size=nb)
        c.local1[:nb, i, :3] = p
        c.local2[:nb, i, :3] = p + rng.normal(scale=0.01, size=(nb, 3))
    z = np.zeros(n, np.int32)
    pairs = A.HostPairs(z, z, np.zeros((n, 4)), q, np.zeros((n, 4)), np.tile([0, 0, 0, 1.0], (n, 1)))
    return pairs, c


# (kind, seed, steps before the captured one, grid nx, ny, nz, variety:
# bit 0 random materials / dampings / locks / kinematic bodies, bit 1
# collision category and mask filters)
DYNAMICS_CASES = [(0, 1, 60, 4, 3, 4, 1), (1, 3, 150, 4, 3, 4, 1), (1, 5, 300, 4, 3, 4, 1), (0, 6, 200, 8, 4, 8, 1),
                  (1, 4, 40, 4, 3, 4, 1), (1, 21, 100, 5, 3, 5, 3)]


def dynamics_fixture():
    d = {}
    for kind, seed, steps, nx, ny, nz, variety in DYNAMICS_CASES:
        w = reflib.RefWorld(kind=kind, seed=seed, nx=nx, ny=ny, nz=nz, variety=variety)
        w.step(n=steps)
        w.apply_forces(seed + 1)
        cap = w.capture()
        name = f"k{kind}_s{seed}_t{steps}"
        for k, v in cap.items():
            d[name + "/" + k] = v
        print(name, "bodies", len(cap["in_body_mass"]), "manifolds", len(cap["in_manifold_ids"]),
              "points", len(cap["in_point_normal_depth"]), "islands", len(cap["in_island_manifold_start"]))
    np.savez_compressed(os.path.join(HERE, "np_dynamics.npz"), **d)


def world_fixture():
    import worldio
    d = {}
    for name in worldio.WORLD_CASES:
        sc, steps, every = worldio.make_scene(name)
        t = worldio.trajectory(reflib.RefScene(sc), steps, every, worldio.DRIVERS.get(name))
        for k, v in t.items():
            d[f"{name}/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "world.npz"), **d)


def main(parts=("scene", "manifold", "dynamics", "world")):
    if parts == ("dynamics",):
        dynamics_fixture()
        return
    if parts == ("world",):
        world_fixture()
        return
    ref = reflib.RefEngine("f32")
    verts, faces = ref.quickhull(scenes.icosphere42_points())
    if "scene" not in parts:
        mesh = ref.create_convex_mesh(verts, faces)
        ref.create_convex_mesh_shape(mesh)
        ref.create_convex_mesh_shape(mesh, edgecases.HULL_SCALE)
        manifold_fixture(ref, verts, faces)
        return
    with open(os.path.join(HERE, "hull42.json"), "w") as fh:
        json.dump({"source": "reference QuickHull of scenes.icosphere42_points(seed=7, radius=0.8, noise=0.05)",
                   "vertices": [[float(x) for x in v] for v in verts], "faces": faces}, fh)
    print("hull:", len(verts), "vertices", len(faces), "faces")

    mesh = ref.create_convex_mesh(verts, faces)
    ref.create_convex_mesh_shape(mesh)                       # instance 0: scale 1
    ref.create_convex_mesh_shape(mesh, edgecases.HULL_SCALE)  # instance 1: scaled

    sc = scenes.narrowphase_scene(total_pairs=7 * 192, seed=11, hull=(verts, faces))
    d = {"shapes": sc.shapes}
    rng = np.random.default_rng(12)
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        pa = pairs.slice(0, pairs.n)
        outa, _ = ref.narrowphase(algo, sc.shapes, pa)
        goldenio.pack_case(d, f"{name}_a_", algo, pairs, outa, pa.cache)
        pb = reflib.perturb_pairs(pa, rng)
        pb.cache = reflib.next_frame_cache(pa.cache, outa)
        pbin = pb.slice(0, pb.n)
        outb, _ = ref.narrowphase(algo, sc.shapes, pb)
        goldenio.pack_case(d, f"{name}_b_", algo, pbin, outb, pb.cache)
        print(name, "colliding a/b:", outa.is_colliding.mean(), outb.is_colliding.mean())
    np.savez_compressed(os.path.join(HERE, "np_scene.npz"), **d)

    shapes, cases = edgecases.build()
    e = {"shapes": shapes}
    for cname, algo, pairs, max_contacts in cases:
        pin = pairs.slice(0, pairs.n)
        out, _ = ref.narrowphase(algo, shapes, pairs, out=A.HostContacts(pairs.n, max_contacts))
        goldenio.pack_case(e, f"{cname}_", algo, pin, out, pairs.cache)
        print(cname, "colliding:", out.is_colliding.tolist(), "contacts:", out.nb_contacts.tolist())
    np.savez_compressed(os.path.join(HERE, "np_edge.npz"), **e)
    if "manifold" in parts:
        manifold_fixture(ref, verts, faces)
    if "dynamics" in parts:
        dynamics_fixture()
    if "world" in parts:
        world_fixture()


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("scene", "manifold", "dynamics", "world"))
