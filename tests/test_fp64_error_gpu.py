"""Error of the GPU narrow phase against the reference's double build.

The GPU is bit-identical to the reference's float build; this test states
how far both are from the reference compiled with
IS_RP3D_DOUBLE_PRECISION_ENABLED (outputs rounded to float) on a seeded
sample of all seven batches of the microbenchmark, with the tolerances the
bench reports against:
  - at least 99.9% of pairs on the same path (same colliding flag and
    contact count);
  - on those pairs, per contact: normal components within 1e-3, depth within
    1e-4 m, local points within 1e-3 m (shapes are 0.2-1 m in size)."""
import numpy as np
import pytest

import reflib
from reactphysics3d_b200 import _abi as A
from reactphysics3d_b200 import engine, scenes

TOL = {"normal": 1e-3, "depth": 1e-4, "point": 1e-3, "same_path": 0.999}

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (reflib.have_ref("f32") and reflib.have_ref("f64")),
                                 reason="reference builds oracle/_ref not present")]


@pytest.fixture(scope="module")
def setup():
    sc = scenes.narrowphase_scene(total_pairs=7 * 4000, seed=2024)
    ctx = engine.Context(0)
    r32, r64 = reflib.RefEngine("f32"), reflib.RefEngine("f64")
    tables = {}
    for name, e in (("gpu", ctx), ("f32", r32), ("f64", r64)):
        inst = e.create_convex_mesh_shape(e.create_convex_mesh(sc.hull_vertices, sc.hull_faces))
        # the reference harness keeps meshes for the whole process: rename
        # instance 0 of the workload's table to the id this registration got
        s = np.array(sc.shapes, copy=True)
        s["mesh"][s["kind"] == A.SHAPE_CONVEX_MESH] = inst
        tables[name] = s
    ctx.set_shapes(tables["gpu"])
    yield sc, ctx, r32, r64, tables
    ctx.close()


@pytest.mark.parametrize("name", scenes.BATCH_NAMES)
def test_error_against_double_build(setup, name):
    sc, ctx, r32, r64, tables = setup
    algo, pairs = sc.batches[name]
    ours = ctx.narrowphase_host(algo, pairs.slice(0, pairs.n))
    f32, _ = r32.narrowphase(algo, tables["f32"], pairs.slice(0, pairs.n), nthreads=4)
    f64, _ = r64.narrowphase(algo, tables["f64"], pairs.slice(0, pairs.n), nthreads=4)
    assert all(v == 0 for v in reflib.compare_contacts(ours, f32, pairs.n).values())
    same = (ours.is_colliding == f64.is_colliding) & (ours.nb_contacts == f64.nb_contacts)
    assert same.mean() >= TOL["same_path"], same.mean()
    mask = ours.valid_mask() & same[None, :]
    assert mask.sum() > 100
    nd = np.abs(ours.normal_depth.astype(np.float64) - f64.normal_depth)[mask]
    assert nd[:, :3].max() <= TOL["normal"], nd[:, :3].max()
    assert nd[:, 3].max() <= TOL["depth"], nd[:, 3].max()
    for f in ("local1", "local2"):
        e = np.abs(getattr(ours, f).astype(np.float64) - getattr(f64, f))[mask][:, :3]
        assert e.max() <= TOL["point"], (f, e.max())
