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


def main():
    ref = reflib.RefEngine("f32")
    verts, faces = ref.quickhull(scenes.icosphere42_points())
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


if __name__ == "__main__":
    main()
