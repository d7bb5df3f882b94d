"""World step on the GPU (rp3dg_world_*, the drop-in for PhysicsWorld::update)
against the reference float build: every step's overlapping pairs in the
reference's array order, the solver's contact manifolds and points, and the
body states (positions, orientations, velocities, sleeping flags) must be
bit-identical."""
import os

import numpy as np
import pytest

import rayio
import reflib
import worldio
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "world.npz")


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    yield c
    c.close()


def fixture(name):
    z = np.load(GOLDEN)
    return {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


@pytest.mark.parametrize("name", list(worldio.WORLD_CASES))
def test_world_matches_reference_fixture(ctx, name):
    sc, steps, every = worldio.make_scene(name)
    w = engine.World(ctx, sc)
    got = worldio.trajectory(w, steps, every, worldio.DRIVERS.get(name))
    exp = fixture(name)
    assert worldio.first_mismatch(got, exp) is None, worldio.first_mismatch(got, exp)
    for k in ("ckpt_pos", "ckpt_ori", "ckpt_lv", "ckpt_av", "ckpt_sleep"):
        assert np.array_equal(got[k], exp[k]), k
    w.close()


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
def test_box_pile_1000_matches_reference_live(ctx):
    """The full plain box pile (1,000 boxes, 300 steps at 1/60 s): pair
    arrays, manifolds and final states bit-identical to the reference."""
    sc = scenes.box_pile()
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    for s in range(300):
        w.update(float(worldio.DT))
        r.update(float(worldio.DT))
        if s % 25 == 24 or s == 299:
            assert np.array_equal(w.pairs(), r.pairs()), s
            cw, cr = w.contacts(), r.contacts()
            for a, b in zip(cw, cr):
                assert np.array_equal(a, b), s
    for a, b in zip(w.bodies(), r.bodies()):
        assert np.array_equal(a, b)
    assert w.bodies()[4].sum() > 0      # some boxes asleep after 5 s
    w.close()


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
def test_single_world_with_device_tree_matches_reference(ctx):
    """A single world switched to a device tree (one GPU thread replaying
    all its reinsertions) and back to the host tree mid-run: the 1,000-box
    pile's pairs, manifolds and states stay bit-identical to the reference,
    and world raycasts (which copy the device tree back) hit what the
    reference hits."""
    sc = scenes.box_pile()
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    assert not w.device_trees
    w.set_device_trees(True)
    rays = scenes.world_rays(3000, (-12, -0.5, -12), (12, 12, 12), seed=8, masks=(0xFFFF,))
    for s in range(160):
        if s == 120:
            w.set_device_trees(False)
        w.update(float(worldio.DT))
        r.update(float(worldio.DT))
        if s % 40 == 39:
            assert np.array_equal(w.pairs(), r.pairs()), s
            for a, b in zip(w.contacts(), r.contacts()):
                assert np.array_equal(a, b), s
            hw, nw = w.raycast(rays, A.RAYCAST_ALL, 4)
            hr, nr = r.raycast(rays, A.RAYCAST_ALL, 4)
            assert rayio.same_hits((hw, nw), (hr, nr)), s
    for a, b in zip(w.bodies(), r.bodies()):
        assert np.array_equal(a, b)
    w.close()


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
def test_terrain_world_matches_reference_live(ctx):
    """400 boxes, spheres and capsules falling onto a 40 x 40 height field
    (300 steps at 1/60 s): the convex vs concave pairs, their triangle tests
    and up to four manifolds per pair give pair arrays, manifolds, points
    and final states bit-identical to the reference."""
    sc = scenes.heightfield_world(n_bodies=400, cols=40, rows=40, seed=21)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    multi = 0
    for s in range(300):
        w.update(float(worldio.DT))
        r.update(float(worldio.DT))
        if s % 25 == 24 or s == 299:
            assert np.array_equal(w.pairs(), r.pairs()), s
            cw, cr = w.contacts(), r.contacts()
            for a, b in zip(cw, cr):
                assert np.array_equal(a, b), s
            b1, b2 = cw[0], cw[1]
            keys = b1.astype(np.int64) * 100000 + b2
            multi = max(multi, len(keys) - len(np.unique(keys)))
    for a, b in zip(w.bodies(), r.bodies()):
        assert np.array_equal(a, b)
    assert multi > 0                    # some terrain pairs carried several manifolds
    assert w.bodies()[4].sum() > 0      # bodies come to rest on the terrain
    w.close()


def largest_island(b1, b2, static=(0,)):
    """Manifolds of the largest island (connected through movable bodies)."""
    par = {}

    def find(x):
        while par.get(x, x) != x:
            x = par[x]
        return x

    for a, b in zip(b1.tolist(), b2.tolist()):
        if a in static or b in static:
            continue
        ra, rb = find(a), find(b)
        if ra != rb:
            par[ra] = rb
    sizes = {}
    for a, b in zip(b1.tolist(), b2.tolist()):
        r = find(a if a not in static else b)
        sizes[r] = sizes.get(r, 0) + 1
    return max(sizes.values()) if sizes else 0


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
def test_island_beyond_shared_memory_matches_reference(ctx):
    """2,500 bodies piling on a 36 x 36 height field form one island of
    thousands of manifolds, too large for a CTA's shared memory: its level
    schedule is built in global memory and its rows are streamed through the
    staging ring.  Pairs, manifolds, points and states stay bit-identical to
    the reference."""
    sc = scenes.heightfield_world(n_bodies=2500, cols=36, rows=36, seed=31)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    big = 0
    for s in range(150):
        w.update(float(worldio.DT))
        r.update(float(worldio.DT))
        if s >= 90 and (s % 10 == 9 or s == 149):
            assert np.array_equal(w.pairs(), r.pairs()), s
            cw, cr = w.contacts(), r.contacts()
            for a, b in zip(cw, cr):
                assert np.array_equal(a, b), s
            big = max(big, largest_island(cw[0], cw[1]))
    for a, b in zip(w.bodies(), r.bodies()):
        assert np.array_equal(a, b)
    assert big >= 2000, big
    w.close()


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
def test_many_moved_colliders_match_reference(ctx):
    """5,000 bodies over a 64 x 64 height field: in the first steps more than
    4,096 colliders move at once, so the broad phase's tree queries run on
    the GPU over a copy of the tree; the pair arrays (whose order follows the
    queries' visiting order), manifolds and states stay bit-identical."""
    sc = scenes.heightfield_world(n_bodies=5000, cols=64, rows=64, seed=41)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    for s in range(40):
        w.update(float(worldio.DT))
        r.update(float(worldio.DT))
        if s < 3 or s % 5 == 4:
            assert np.array_equal(w.pairs(), r.pairs()), s
            cw, cr = w.contacts(), r.contacts()
            for a, b in zip(cw, cr):
                assert np.array_equal(a, b), s
    assert w.stats()["moved_colliders"] >= 4096
    for a, b in zip(w.bodies(), r.bodies()):
        assert np.array_equal(a, b)
    w.close()


def test_heightfield_rejects_bad_input(ctx):
    with pytest.raises(engine.Rp3dgError):
        ctx.create_heightfield(np.zeros((1, 5), np.float32))          # fewer than two rows
    with pytest.raises(engine.Rp3dgError):
        ctx.create_heightfield(np.zeros((4, 4), np.float32), scale=(1.0, 0.0, 1.0))
    sc = scenes.heightfield_world(n_bodies=4, cols=8, rows=8)
    bad = scenes.WorldScene(sc.settings, sc.shapes, sc.bodies.copy(), sc.colliders, heightfields=sc.heightfields)
    bad.bodies["type"][0] = A.BODY_DYNAMIC
    with pytest.raises(engine.Rp3dgError):
        engine.World(ctx, bad)          # a height field must be on a static body


def test_world_create_rejects_bad_input(ctx):
    sc = scenes.box_pile(2, 2, 2)
    bad = scenes.WorldScene(sc.settings, sc.shapes, sc.bodies, sc.colliders[::-1].copy())
    with pytest.raises(engine.Rp3dgError):
        engine.World(ctx, bad)          # colliders not grouped by ascending body
    bad = scenes.WorldScene(sc.settings, sc.shapes, sc.bodies, sc.colliders.copy())
    bad.colliders["shape"][3] = len(sc.shapes) + 5
    with pytest.raises(engine.Rp3dgError):
        engine.World(ctx, bad)          # shape outside the table
    w = engine.World(ctx, sc)
    with pytest.raises(engine.Rp3dgError):
        w.update(0.0)                    # dt must be positive
    w.close()


def test_world_stats_and_launches(ctx):
    sc = scenes.box_pile(4, 4, 4, seed=2)
    w = engine.World(ctx, sc)
    l0 = ctx.kernel_launches()
    w.update(float(worldio.DT), 90)
    st = w.stats()
    assert st["contact_pairs"] > 0 and st["manifolds"] == st["contact_pairs"]
    assert st["overlapping_pairs"] >= st["contact_pairs"]
    assert ctx.kernel_launches() - l0 >= 90 * 5
    w.close()


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
def test_world_group_matches_each_reference_world(ctx):
    """Worlds of different kinds and sizes stepped together in one group (and
    on several host threads) each stay bit-identical to their own reference
    world: pair arrays, manifolds and states at every step."""
    parts = [scenes.mixed_world(4, 3, 4, seed=11), scenes.box_pile(3, 4, 3, seed=12),
             scenes.ragdoll_world(2, seed=15, limits=False, boxes=3),
             scenes.mixed_world(3, 3, 3, seed=13, variety=False)]
    many = scenes.many_worlds(3, seed=14, min_bodies=20, max_bodies=60, merge=False, limits=False)
    shapes, merged = scenes.merge_shapes(parts + many)
    g = engine.WorldGroup(ctx, merged, shapes, threads=4)
    refs = [reflib.RefScene(s) for s in parts + many]
    for step in range(150):
        g.update(float(worldio.DT))
        for k, r in enumerate(refs):
            r.update(float(worldio.DT))
            if step % 10 == 9:
                assert np.array_equal(g.pairs(k), r.pairs()), (step, k)
                for a, b in zip(g.contacts(k), r.contacts()):
                    assert np.array_equal(a, b), (step, k)
                for a, b in zip(g.bodies(k), r.bodies()):
                    assert np.array_equal(a, b), (step, k)
    st = g.stats()
    assert st["manifolds"] > 0
    g.close()


def test_autotuned_scheduling_gives_identical_results(ctx):
    """The autotuner varies which kernel takes which island and how many
    persistent CTAs run; the results must not depend on it: a group tuned
    over its first steps ends bit-identical to the same group untuned, and
    the chosen setting is one of the candidates."""
    shapes, scs = scenes.many_worlds(96, seed=21, min_bodies=20, max_bodies=200, ragdolls=(1, 2), limits=True)
    a = engine.WorldGroup(ctx, scs, shapes, threads=4)
    b = engine.WorldGroup(ctx, scs, shapes, threads=4)
    a.autotune(rounds=1)
    assert a.tuning()["tuning"]
    for _ in range(40):
        a.update(float(worldio.DT))
        b.update(float(worldio.DT))
    t = a.tuning()
    assert not t["tuning"]
    assert t["small_max"] in (4, 8, 16, 32) and t["giant_min"] in (128, 256, 512) and t["large_per_sm"] in (1, 2)
    for k in range(len(scs)):
        for x, y in zip(a.bodies(k), b.bodies(k)):
            assert np.array_equal(x, y), k
    a.close()
    b.close()


def test_device_trees_give_identical_results(ctx):
    """A world group keeps its broad-phase trees on the device (reinsertions
    one GPU thread per world, queries one thread per moved collider); the
    same group with host trees, and one switched between the two every few
    steps, end with the same pairs, contacts and states at every checkpoint,
    and world raycasts (which copy a world's device tree back) hit the same
    colliders at the same points."""
    shapes, scs = scenes.many_worlds(96, seed=23, min_bodies=20, max_bodies=200, ragdolls=(1, 2), limits=True)
    a = engine.WorldGroup(ctx, scs, shapes, threads=4)
    b = engine.WorldGroup(ctx, scs, shapes, threads=4)
    c = engine.WorldGroup(ctx, scs, shapes, threads=4)
    assert a.device_trees and b.device_trees
    b.set_device_trees(False)
    assert not b.device_trees
    rays = scenes.world_rays(4000, (-12, -0.5, -12), (12, 8, 12), seed=5, masks=(0xFFFF,))
    for step in range(60):
        for g in (a, b, c):
            g.update(float(worldio.DT))
        if step % 7 == 3:
            c.set_device_trees(not c.device_trees)
        if step % 15 == 14:
            for k in (0, 17, 50, 95):
                pa = a.pairs(k)
                assert np.array_equal(pa, b.pairs(k)) and np.array_equal(pa, c.pairs(k)), (step, k)
                for x, y, z in zip(a.contacts(k), b.contacts(k), c.contacts(k)):
                    assert np.array_equal(x, y) and np.array_equal(x, z), (step, k)
                for x, y in zip(a.bodies(k), b.bodies(k)):
                    assert np.array_equal(x, y), (step, k)
                ha, na = a.raycast(rays, A.RAYCAST_ALL, 4, world=k)
                hb, nb = b.raycast(rays, A.RAYCAST_ALL, 4, world=k)
                assert np.array_equal(na, nb) and np.array_equal(ha, hb), (step, k)
    assert a.stats()["overlapping_pairs"] > 0
    one = engine.World(ctx, scs[0])
    assert not one.device_trees
    for g in (a, b, c, one):
        g.close()


def test_groups_on_two_contexts_step_concurrently(ctx):
    """Two world groups, each on its own context, stepped at the same time
    from two host threads (the library's host bookkeeping and its streams
    are per context), end bit-identical to one group holding all the
    worlds."""
    import threading
    raw = scenes.many_worlds(64, seed=29, min_bodies=20, max_bodies=120, ragdolls=(1, 2), merge=False)
    shapes, scs = scenes.merge_shapes(raw)
    one = engine.WorldGroup(ctx, scs, shapes, threads=4)
    parts = []
    for lo, hi in ((0, 30), (30, 64)):
        c = engine.Context(0)
        sh, sc = scenes.merge_shapes(raw[lo:hi])
        parts.append((c, engine.WorldGroup(c, sc, sh, threads=2), lo))
    dt = float(worldio.DT)
    ths = [threading.Thread(target=g.update, args=(dt, 80)) for _, g, _ in parts]
    [t.start() for t in ths]
    one.update(dt, 80)
    [t.join() for t in ths]
    for k in range(64):
        c, g, lo = parts[0] if k < 30 else parts[1]
        for x, y in zip(one.bodies(k), g.bodies(k - lo)):
            assert np.array_equal(x, y), k
        assert np.array_equal(one.pairs(k), g.pairs(k - lo)), k
    one.close()
    for c, g, _ in parts:
        g.close()
        c.close()


@pytest.mark.skipif(not (reflib.have_ref("f32") and reflib.have_ref("f64")), reason="reference engine not built")
def test_ragdolls_with_limits_stay_within_tolerance(ctx):
    """Cone and hinge limits go through acos / atan2, whose last bit differs
    between CUDA and the host C library, so ragdolls with limits are compared
    within a tolerance, the one the reference itself shows between its float
    and double builds: over the first 30 steps (the limits engage, the bodies
    hit the ground and each other) the largest position difference from the
    float reference stays within the largest difference between the
    reference's float and double builds; after 240 steps every body rests
    above the ground."""
    sc = scenes.ragdoll_world(4, seed=29, limits=True, boxes=4)
    w, r, r64 = engine.World(ctx, sc), reflib.RefScene(sc), reflib.RefScene(sc, "f64")
    ours, spread = 0.0, 0.0
    for s in range(240):
        w.update(float(worldio.DT))
        r.update(float(worldio.DT))
        if s < 30:
            r64.update(float(worldio.DT))
            pr = r.bodies()[0].astype(np.float64)
            ours = max(ours, float(np.abs(w.bodies()[0] - pr).max()))
            spread = max(spread, float(np.abs(r64.bodies()[0] - pr).max()))
    assert ours <= max(spread, 1e-5), (ours, spread)
    pw, pr = w.bodies()[0], r.bodies()[0]
    assert (pw[1:, 1] > 0.45).all() and (pr[1:, 1] > 0.45).all()
    w.close()


def _slider_translations(bodies, n):
    """Translation of each mechanism's sliding box along its slider from the
    creation offset (positions of bodies 8 and 9 of each 12-body mechanism)."""
    p = bodies[0].astype(np.float64)
    return np.array([p[9 + 12 * m, 1] - p[8 + 12 * m, 1] - 2.1 for m in range(n)])


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
def test_mechanisms_match_reference_live(ctx):
    """Fixed and slider joints (translation limits, a motor whose speed is set
    before every step) next to ball-and-socket chains and motorised hinges:
    36 copies of the testbed's joints scene stay bit-identical to the float
    reference for 300 steps (pairs, manifolds and states every 10 steps), and
    the sliders reach both of their limits."""
    n = 36
    sc = scenes.mechanism_world(n, seed=37)
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    lo, hi = np.inf, -np.inf
    for s in range(300):
        for j, v in scenes.mechanism_motor_speeds(n, s, worldio.DT):
            w.set_motor_speed(j, v)
            r.set_motor_speed(j, v)
        w.update(float(worldio.DT))
        r.update(float(worldio.DT))
        if s % 10 == 9:
            assert np.array_equal(w.pairs(), r.pairs()), s
            for a, b in zip(w.contacts(), r.contacts()):
                assert np.array_equal(a, b), s
            for a, b in zip(w.bodies(), r.bodies()):
                assert np.array_equal(a, b), s
            u = _slider_translations(r.bodies(), n)
            lo, hi = min(lo, u.min()), max(hi, u.max())
    assert lo < -1.6 and hi > 1.6, (lo, hi)
    w.close()


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
def test_mechanism_group_matches_reference_worlds(ctx):
    """Mechanism worlds in one group, motor speeds set per world: each world
    stays bit-identical to its own reference world."""
    parts = [scenes.mechanism_world(k, seed=40 + k) for k in (1, 3, 2)]
    shapes, merged = scenes.merge_shapes(parts)
    g = engine.WorldGroup(ctx, merged, shapes, threads=2)
    refs = [reflib.RefScene(s) for s in parts]
    for s in range(150):
        for k, (part, r) in enumerate(zip((1, 3, 2), refs)):
            for j, v in scenes.mechanism_motor_speeds(part, s, worldio.DT):
                g.set_motor_speed(j, v, world=k)
                r.set_motor_speed(j, v)
        g.update(float(worldio.DT))
        for k, r in enumerate(refs):
            r.update(float(worldio.DT))
            if s % 10 == 9:
                for a, b in zip(g.bodies(k), r.bodies()):
                    assert np.array_equal(a, b), (s, k)
    g.close()


def test_motor_speed_rejects_bad_joints(ctx):
    sc = scenes.mechanism_world(1)
    w = engine.World(ctx, sc)
    with pytest.raises(engine.Rp3dgError):
        w.set_motor_speed(0, 1.0)        # a ball-and-socket joint has no motor
    with pytest.raises(engine.Rp3dgError):
        w.set_motor_speed(8, 1.0)        # nor has a fixed joint
    with pytest.raises(engine.Rp3dgError):
        w.set_motor_speed(len(sc.joints), 1.0)
    w.set_motor_speed(6, 0.5)            # the slider
    w.set_motor_speed(7, -1.0)           # the hinge
    w.update(float(worldio.DT))
    w.close()


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference engine not built")
@pytest.mark.parametrize("name,make,steps", [
    ("mixed", lambda: scenes.mixed_world(5, 4, 5, seed=5), 300),
    ("hulls", lambda: scenes.hull_world(4, 3, 4, seed=44), 200),
    ("terrain", lambda: scenes.heightfield_world(n_bodies=80, cols=20, rows=20, seed=45), 200),
    ("mechanisms", lambda: scenes.mechanism_world(4, seed=46), 200),
])
def test_contact_events_match_reference(ctx, name, make, steps):
    """EventListener::onContact after every update: the contact pairs in
    creation order with ContactStart / ContactStay, then the lost pairs with
    ContactExit (removed by the broad phase or no longer touching), and each
    pair's contact points, bit-identical to the reference; every kind of
    event occurs (in the mechanisms, whose joined bodies do not collide,
    contacts are rare)."""
    sc = make()
    w, r = engine.World(ctx, sc), reflib.RefScene(sc)
    seen = np.zeros(3, np.int64)
    for s in range(steps):
        if name == "mechanisms":
            for j, v in scenes.mechanism_motor_speeds(4, s, worldio.DT):
                w.set_motor_speed(j, v)
                r.set_motor_speed(j, v)
        w.update(float(worldio.DT))
        r.update(float(worldio.DT))
        got, exp = w.contact_events(), r.contact_events()
        assert got[0].tobytes() == exp[0].tobytes(), (s, len(got[0]), len(exp[0]))
        for a, b in zip(got[1:], exp[1:]):
            assert np.array_equal(a, b), s
        seen += np.bincount(got[0]["type"], minlength=3)[:3]
    # joint-connected bodies do not collide: the mechanisms touch rarely
    assert (seen > 0).all() if name != "mechanisms" else seen.sum() > 0, seen
    w.close()
