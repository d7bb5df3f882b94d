"""Dynamics stage on the GPU (rp3dg_dynamics_step_host / _device through the
C ABI) against the reference's own outputs (committed fixture), bit-exact;
thousands of worlds in one call; input validation."""
import ctypes as C

import numpy as np
import pytest

import dynio
import reflib
from reactphysics3d_b200 import dynamics as D
from reactphysics3d_b200 import engine

pytestmark = pytest.mark.gpu
GOLDEN = reflib.ROOT + "/tests/golden/np_dynamics.npz"


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    c = engine.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def fixture():
    return np.load(GOLDEN)


@pytest.mark.parametrize("api", ["host", "device"])
def test_gpu_matches_reference_fixture(ctx, fixture, api):
    for n in dynio.cases(fixture):
        cap = dynio.capture(fixture, n)
        w = D.world_from_capture(cap)
        if api == "device":
            w = D.DynWorld(w.a, w.nb_enabled, w.nc_enabled, device="cuda")
        ctx.dynamics_step(D.params_from_capture(cap), w)
        ctx.synchronize()
        assert dynio.mismatches(w, cap) == {}, (n, api)
    assert ctx.device_errors(clear=True) & 4 == 0


def test_gpu_many_worlds(ctx, fixture):
    """6,000 worlds (1,200 copies of each fixture world, about 100k bodies and
    100k manifolds) in one device call: every world equals the reference's
    result for that world, and a second run is bit-identical."""
    caps = [dynio.capture(fixture, n) for n in dynio.cases(fixture)]
    worlds = [D.world_from_capture(c) for c in caps]
    reps = 1200
    batch, layout = D.batch_worlds(worlds * reps)
    params = D.params_from_capture(caps[0])
    dev = D.DynWorld(batch.a, batch.nb_enabled, batch.nc_enabled, device="cuda")
    dev2 = D.DynWorld(batch.a, batch.nb_enabled, batch.nc_enabled, device="cuda")
    ctx.dynamics_step(params, dev)
    ctx.dynamics_step(params, dev2)
    ctx.synchronize()
    h, h2 = dev.host(), dev2.host()
    for k in D.OUTPUTS:
        assert np.array_equal(np.asarray(h[k]).view(np.uint8), np.asarray(h2[k]).view(np.uint8)), k
    out = D.unbatch_worlds(h, layout)
    rng = np.random.default_rng(3)
    for j in rng.choice(len(out), size=300, replace=False):
        assert dynio.mismatches(out[j], caps[j % len(caps)]) == {}, j
    assert ctx.device_errors(clear=True) & 4 == 0


def test_gpu_dynamics_errors(ctx, fixture):
    cap = dynio.capture(fixture, dynio.cases(fixture)[0])
    params = D.params_from_capture(cap)
    # misaligned float4 array: refused on the host before any launch
    w = D.DynWorld(D.world_from_capture(cap).a, int(cap["in_body_nb_enabled"][0]),
                   int(cap["in_collider_nb_enabled"][0]), device="cuda")
    b, c, m, p, i = w.structs()
    b.linear_velocity = w["linear_velocity"].data_ptr() + 4
    rc = ctx.lib.rp3dg_dynamics_step_device(ctx.h, C.byref(params), C.byref(b), C.byref(c), C.byref(m), C.byref(p),
                                            C.byref(i))
    assert rc == -1 and b"misaligned" in ctx.lib.rp3dg_last_error(ctx.h)
    # a manifold naming a body outside the table and an island past the end:
    # skipped by the kernels, error bit 2 set, the rest still solved
    a = dict(D.world_from_capture(cap).a)
    ids = np.array(a["ids"]).reshape(-1, 4)
    ids[0, 1] = 10_000
    a["ids"] = ids
    a["manifold_count"] = np.array(a["manifold_count"])
    a["manifold_count"][-1] = 1_000_000
    bad = D.DynWorld(a, int(cap["in_body_nb_enabled"][0]), int(cap["in_collider_nb_enabled"][0]), device="cuda")
    assert ctx.device_errors(clear=True) == 0
    ctx.dynamics_step(params, bad)
    ctx.synchronize()
    assert ctx.device_errors(clear=True) & 4
    bad_p = D.make_params(dt=0.0)
    with pytest.raises(engine.Rp3dgError):
        ctx.dynamics_step(bad_p, D.world_from_capture(cap))
