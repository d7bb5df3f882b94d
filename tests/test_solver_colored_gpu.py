"""Graph-coloured contact solver of the world step (rp3dg_world_set_solver,
RP3DG_SOLVER_GRAPH_COLORED): not the drop-in, so it is held to physical
checks next to the exact-order solver on the same world instead of bit
equality with the reference:
  - turning the statistics on does not change the exact solver's results;
  - the coloured solver is deterministic (two runs give the same states);
  - it colours with few colours, its velocity constraint residual stays of
    the exact solver's order, and the pile comes to rest (the energy only
    drifts down)."""
import numpy as np
import pytest

from reactphysics3d_b200 import engine, scenes

pytestmark = pytest.mark.gpu
DT = float(np.float32(1.0 / 60.0))


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    yield c
    c.close()


def _run(ctx, sc, steps, solver, stats):
    w = engine.World(ctx, sc)
    w.set_solver(solver, stats)
    trace = []
    for _ in range(steps):
        w.update(DT)
        if stats:
            trace.append(w.solver_stats())
    out = w.bodies()
    w.close()
    return out, trace


def test_stats_do_not_change_the_exact_solver(ctx):
    sc = scenes.box_pile(nx=4, ny=4, nz=4, seed=3)
    a, _ = _run(ctx, sc, 90, engine.SOLVER_EXACT, False)
    b, trace = _run(ctx, sc, 90, engine.SOLVER_EXACT, True)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert trace[-1]["contact_points"] > 0 and trace[-1]["colors"] == 0


def test_colored_solver_is_deterministic_and_settles(ctx):
    sc = scenes.box_pile(nx=5, ny=5, nz=5, seed=3)
    steps = 240
    exact, te = _run(ctx, sc, steps, engine.SOLVER_EXACT, True)
    col, tc = _run(ctx, sc, steps, engine.SOLVER_GRAPH_COLORED, True)
    col2, _ = _run(ctx, sc, steps, engine.SOLVER_GRAPH_COLORED, True)
    assert all(np.array_equal(x, y) for x, y in zip(col, col2))
    # different order, different floats
    assert not all(np.array_equal(x, y) for x, y in zip(col, exact))
    active = [t for t in tc if t["contact_points"] > 0]
    assert active and all(1 <= t["colors"] <= 128 for t in active)
    assert max(t["colors"] for t in active) <= 32
    # residual of the same order as the exact solver's, over the resting phase
    rc = np.mean([t["residual_rms"] for t in tc[-60:]])
    re = np.mean([t["residual_rms"] for t in te[-60:]])
    assert np.isfinite(rc) and rc <= 4.0 * re + 1e-3, (rc, re)
    # the pile comes to rest: little kinetic energy left, total energy not above its start
    e0 = tc[0]["kinetic_energy"] + tc[0]["potential_energy"]
    e = np.array([t["kinetic_energy"] + t["potential_energy"] for t in tc])
    assert np.all(e <= e0 + 1e-3 * abs(e0) + 1.0)
    assert tc[-1]["kinetic_energy"] < 0.1 * max(t["kinetic_energy"] for t in tc)
    # the pile is chaotic and the colour order is not the exact one, so the
    # bodies end in different places; the pile as a whole rests at a similar
    # height (mean resting height within a third of a box size)
    hy_c, hy_e = float(np.mean(col[0][:, 1])), float(np.mean(exact[0][:, 1]))
    assert abs(hy_c - hy_e) < 0.35, (hy_c, hy_e)


def test_bad_solver_is_rejected(ctx):
    w = engine.World(ctx, scenes.box_pile(nx=2, ny=2, nz=2, seed=1))
    with pytest.raises(engine.Rp3dgError):
        w.set_solver(7)
    w.close()
