"""The narrow-phase workload at its full size against the reference build
itself: all 1,048,576 pairs of the seven batches (the bench's seeded scene),
a first frame with fresh temporal-coherence caches and a second frame with
moved poses and the first frame's caches, every pair's flags, contact
count, normals, depths, local points and cache bit-identical to the
reference's testCollision (oracle/_ref, run on the host cores)."""
import os

import numpy as np
import pytest

import edgecases
import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build absent")]


def _hulls(e):
    v, f = edgecases.load_hull()
    m = e.create_convex_mesh(v, f)
    return e.create_convex_mesh_shape(m), e.create_convex_mesh_shape(m, edgecases.HULL_SCALE)


def _same(got, exp, cg, ce, what):
    mism = reflib.compare_contacts(got, exp, exp.n)
    assert all(v == 0 for v in mism.values()), (what, mism)
    a = np.ascontiguousarray(cg).view(np.uint8).reshape(-1, 16)
    b = np.ascontiguousarray(ce).view(np.uint8).reshape(-1, 16)
    assert np.array_equal(a, b), (what, "cache", np.argwhere((a != b).any(axis=1))[:5].ravel())


def test_full_workload_matches_reference_two_frames(cuda_lib):
    ctx = engine.Context(0)
    ref = reflib.RefEngine("f32")
    threads = max(1, os.cpu_count() or 1)
    sc = scenes.narrowphase_scene(seed=1234, hull=edgecases.load_hull())
    assert sc.n_pairs == scenes.TOTAL_PAIRS
    ids_g = _hulls(ctx)
    ids_r = _hulls(ref)
    shapes_g = np.array(sc.shapes, copy=True)
    shapes_r = np.array(sc.shapes, copy=True)
    conv = shapes_g["kind"] == A.SHAPE_CONVEX_MESH
    shapes_g["mesh"][conv] = np.asarray(ids_g)[sc.shapes["mesh"][conv]]
    shapes_r["mesh"][conv] = np.asarray(ids_r)[sc.shapes["mesh"][conv]]
    ctx.set_shapes(shapes_g)
    rng = np.random.default_rng(9)
    colliding = 0
    for name, (algo, pairs) in sc.batches.items():
        pairs.cache = A.fresh_cache(pairs.n)
        pg, pr = pairs.slice(0, pairs.n), pairs.slice(0, pairs.n)
        a, _ = ref.narrowphase(algo, shapes_r, pr, nthreads=threads)
        g = ctx.narrowphase_host(algo, pg)
        _same(g, a, pg.cache, pr.cache, name + " frame 1")
        colliding += int(a.is_colliding.sum())
        nxt = reflib.perturb_pairs(pr, rng)
        nxt.cache = reflib.next_frame_cache(pr.cache, a)
        pg2, pr2 = nxt.slice(0, nxt.n), nxt.slice(0, nxt.n)
        a2, _ = ref.narrowphase(algo, shapes_r, pr2, nthreads=threads)
        g2 = ctx.narrowphase_host(algo, pg2)
        _same(g2, a2, pg2.cache, pr2.cache, name + " frame 2")
    assert colliding > 100000
    ctx.close()
