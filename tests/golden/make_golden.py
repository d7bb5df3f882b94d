"""Regenerates the golden fixtures under tests/golden/ from the reference
engine itself (oracle/_ref/librp3d_ref_f32.so, built by `make -C oracle ref`
from the reference's own sources).  Run from the repository root:

    python tests/golden/make_golden.py

Writes:
  hull42.json        the reference QuickHull of the seeded 42-point icosphere
                     (the convex hull used by the hull-box workload)
  np_small.npz       a small seeded narrow-phase scene (all seven batches) with
                     the reference's raw per-pair outputs, fresh caches
  np_coherence.npz   the same scene stepped twice: second pass with slightly
                     moved poses and the caches written by the first pass
                     (temporal-coherence paths of SAT and GJK)
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
import reflib  # noqa: E402


def main():
    ref = reflib.RefEngine("f32")
    verts, faces = ref.quickhull(scenes.icosphere42_points())
    with open(os.path.join(HERE, "hull42.json"), "w") as fh:
        json.dump({"source": "reference QuickHull of scenes.icosphere42_points(seed=7, radius=0.8, noise=0.05)",
                   "vertices": [[float(x) for x in v] for v in verts], "faces": faces}, fh)
    print("hull:", len(verts), "vertices", len(faces), "faces", sorted(set(len(f) for f in faces)))


if __name__ == "__main__":
    main()
