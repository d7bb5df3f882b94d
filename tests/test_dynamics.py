"""Dynamics stage of a world step, CPU side: the C restatement
(rp3do_dynamics_step) against the reference's own phases
(updateBodiesInverseWorldInertiaTensors, integrateRigidBodiesVelocities,
ContactSolverSystem init / warmStart / solve / storeImpulses,
integrateRigidBodiesPositions, updateBodiesState), bit-exact, through the
committed fixture and live; world batching; island independence."""
import numpy as np
import pytest

import dynio
import reflib
from reactphysics3d_b200 import dynamics as D

GOLDEN = reflib.ROOT + "/tests/golden/np_dynamics.npz"


@pytest.fixture(scope="module")
def fixture():
    return np.load(GOLDEN)


def test_fixture_covers_the_paths(fixture):
    names = dynio.cases(fixture)
    assert len(names) >= 4
    tot = {"resting": 0, "new": 0, "kinematic": 0, "locked": 0, "restitution_cases": 0}
    for n in names:
        cap = dynio.capture(fixture, n)
        r = cap["in_point_is_resting"]
        tot["resting"] += int(r.sum())
        tot["new"] += int((r == 0).sum())
        m = cap["in_body_mass"]
        ne = int(cap["in_body_nb_enabled"][0])
        tot["kinematic"] += int(np.sum(m[:ne, 1] == 0))
        tot["locked"] += int(np.sum(np.any(cap["in_body_linear_lock"][:ne, :3] != 1, axis=1)))
    assert all(v > 0 for k, v in tot.items() if k != "restitution_cases"), tot


def test_oracle_matches_reference_fixture(port, fixture):
    for n in dynio.cases(fixture):
        cap = dynio.capture(fixture, n)
        w = D.world_from_capture(cap)
        dynio.run_oracle(port.lib, D.params_from_capture(cap), w)
        assert dynio.mismatches(w, cap) == {}, n


def test_batched_worlds_match_each_world(port, fixture):
    """Several worlds in one call (bodies reordered, indices remapped) give
    each world's reference result: islands of different worlds are
    independent."""
    caps = [dynio.capture(fixture, n) for n in dynio.cases(fixture)]
    worlds = [D.world_from_capture(c) for c in caps] * 2
    params = D.params_from_capture(caps[0])
    assert all(np.array_equal(c["params"], caps[0]["params"]) for c in caps)
    batch, layout = D.batch_worlds(worlds)
    dynio.run_oracle(port.lib, params, batch)
    for w, cap in zip(D.unbatch_worlds(batch, layout), caps * 2):
        assert dynio.mismatches(w, cap) == {}


def test_empty_world(port):
    z4 = np.zeros((0, 4), np.float32)
    a = {f: z4 for f in D.BODY_F4 + ("inv_inertia_world", "local_position", "local_orientation", "world_position",
                                     "world_orientation", "material", "friction_vector1", "friction_vector2",
                                     "friction_impulse", "normal_depth", "local1", "local2")}
    a.update({"gravity": np.zeros(0), "body": np.zeros(0), "ids": np.zeros((0, 4)), "point_start": np.zeros(0),
              "nb_points": np.zeros(0), "penetration_impulse": np.zeros(0), "is_resting": np.zeros(0),
              "manifold_start": np.zeros(0), "manifold_count": np.zeros(0)})
    dynio.run_oracle(port.lib, D.make_params(), D.DynWorld(a, 0, 0))


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build oracle/_ref not present")
@pytest.mark.parametrize("kind,seed,steps", [(0, 11, 90), (1, 12, 200), (1, 13, 20)])
def test_oracle_matches_reference_live(port, kind, seed, steps):
    w = reflib.RefWorld(kind=kind, seed=seed, nx=5, ny=3, nz=5)
    w.step(n=steps)
    w.apply_forces(seed)
    cap = w.capture()
    world = D.world_from_capture(cap)
    dynio.run_oracle(port.lib, D.params_from_capture(cap), world)
    assert dynio.mismatches(world, cap) == {}
