"""Event-counting build of the narrow-phase kernels (the FP32 roofline's path
counters, rp3dg_narrowphase_count_events) on the GPU: it gives the product
kernels' results bit for bit, its counts are those of the reference's code
path (the warp-per-pair and thread-per-pair schedules count the same events
for the same pairs), and simple paths count what they must."""
import numpy as np
import pytest

import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes
from reactphysics3d_b200 import roofline as RF

pytestmark = pytest.mark.gpu
E = {n: k for k, n in enumerate(RF.EVENTS)}


@pytest.fixture(scope="module")
def setup():
    sc = scenes.narrowphase_scene(total_pairs=7 * 2048, seed=77)
    ctx = engine.Context(0)
    m = ctx.create_convex_mesh(sc.hull_vertices, sc.hull_faces)
    ctx.create_convex_mesh_shape(m)
    ctx.set_shapes(sc.shapes)
    yield sc, ctx
    ctx.close()


def _run(ctx, algo, pairs, count):
    dp = engine.DevicePairs(pairs, device="cuda:0")
    out = engine.DeviceContacts(pairs.n, device="cuda:0")
    ev = ctx.narrowphase_count_events(algo, dp, out) if count else None
    if not count:
        ctx.narrowphase_device(algo, dp, out)
    ctx.synchronize()
    return ev, out.to_host(), dp.host_cache()


@pytest.mark.parametrize("name", scenes.BATCH_NAMES)
def test_counting_build_gives_the_same_results(setup, name):
    sc, ctx = setup
    algo, pairs = sc.batches[name]
    for frame in range(2):
        p = pairs.slice(0, pairs.n)
        p.cache = A.fresh_cache(p.n) if frame == 0 else cache
        q = p.slice(0, p.n)
        q.cache = p.cache.copy()
        ev, got, c1 = _run(ctx, algo, p, True)
        _, exp, c2 = _run(ctx, algo, q, False)
        assert all(v == 0 for v in reflib.compare_contacts(got, exp, p.n).values()), name
        assert np.array_equal(c1.view(np.uint8), c2.view(np.uint8))
        assert ev.sum() > 0 and np.all(ev[len(RF.EVENTS):] == 0)
        cache = reflib.next_frame_cache(c1, got)


def test_closed_form_counts(setup):
    sc, ctx = setup
    for name in ("sphere_sphere", "sphere_capsule", "capsule_capsule"):
        algo, pairs = sc.batches[name]
        ev, out, _ = _run(ctx, algo, pairs.slice(0, pairs.n), True)
        assert ev[E["closed_form"]] == pairs.n
        assert ev[E["closed_form_contact"]] == int(out.nb_contacts.sum())
        assert RF.named(ev).keys() == {"closed_form", "closed_form_contact"}


def test_polyhedron_counts_are_bounded(setup):
    sc, ctx = setup
    algo, pairs = sc.batches["box_box"]
    p = pairs.slice(0, pairs.n)
    p.cache = A.fresh_cache(p.n)
    ev, out, _ = _run(ctx, algo, p, True)
    n = pairs.n
    assert ev[E["poly_setup"]] == n
    assert n <= ev[E["face_test"]] <= 12 * n
    assert ev[E["support_box"]] == ev[E["face_test"]]
    assert ev[E["gauss"]] <= 144 * n and ev[E["edge_dist"]] <= ev[E["gauss"]]
    # every colliding pair ends with a face clip or an edge contact
    assert ev[E["clip_setup"]] + ev[E["edge_contact"]] >= int(out.is_colliding.sum())
    assert ev[E["contact"]] + ev[E["edge_contact"]] >= int(out.nb_contacts.sum())


def test_warp_and_thread_schedules_count_the_same_path(setup):
    """Box-box pairs run one per thread in tiles of 32 box-box pairs and one
    per warp in a tile that holds a convex mesh.  Interleaving one hull-box
    pair into every tile sends the box-box pairs through the warp schedule;
    their events (the mixed batch minus the hull pairs alone) must equal
    those of the same pairs on the thread schedule."""
    sc, ctx = setup
    algo, boxes = sc.batches["box_box"]
    _, hulls = sc.batches["hull_box"]
    nb = (boxes.n // 31) * 31
    nt = nb // 31
    bi = np.arange(nb)
    hi = np.arange(nt)

    def pick(src, idx):
        q = src.slice(0, src.n)
        return A.HostPairs(q.shape1[idx], q.shape2[idx], q.pos1[idx], q.rot1[idx], q.pos2[idx], q.rot2[idx])

    b = pick(boxes, bi)
    h = pick(hulls, hi)
    order = []
    for t in range(nt):
        order.append(("h", t))
        order += [("b", t * 31 + k) for k in range(31)]
    cat = lambda f: np.stack([getattr(h, f)[i] if s == "h" else getattr(b, f)[i] for s, i in order])
    mixed = A.HostPairs(cat("shape1"), cat("shape2"), cat("pos1"), cat("rot1"), cat("pos2"), cat("rot2"))
    ev_b, _, _ = _run(ctx, algo, b, True)
    ev_h, _, _ = _run(ctx, algo, h, True)
    ev_m, _, _ = _run(ctx, algo, mixed, True)
    assert np.array_equal(ev_m.astype(np.int64) - ev_h.astype(np.int64), ev_b.astype(np.int64)), \
        (RF.named(ev_m - ev_h), RF.named(ev_b))
