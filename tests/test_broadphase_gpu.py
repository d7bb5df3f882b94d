"""Broad phase on the GPU (rp3dg_broadphase_update_device,
rp3dg_broadphase_pairs_device / _host) against the reference's own broad
phase (committed fixture): bit-exact fat AABBs and reinsertions, identical
pair sets; random AABB sets against the brute-force oracle with the LBVH and
on every sweep axis; thousands of worlds as groups."""
import numpy as np
import pytest
import torch

import bpio
import dynio
import reflib
from reactphysics3d_b200 import broadphase as BP
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


T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_gpu_update_matches_reference(ctx, fixture):
    for n in dynio.cases(fixture):
        cap = dynio.capture(fixture, n)
        ctx.set_shapes(bpio.shapes(cap))
        u = bpio.update_case(cap)
        m = len(u["shape"])
        shape, wpos, wori = T(u["shape"]), T(u["wpos"]), T(u["wori"])
        fmin, fmax = T(u["fat_min"]), T(u["fat_max"])
        moved = torch.full((m,), 7, dtype=torch.uint8, device="cuda")
        bp = BP.make(m, m, 0, shape=shape, world_position=wpos, world_orientation=wori, fat_min=fmin, fat_max=fmax,
                     moved=moved)
        ctx.broadphase_update(bp)
        ctx.synchronize()
        assert np.array_equal(fmin.cpu().numpy().view(np.uint32), u["exp_min"].view(np.uint32)), n
        assert np.array_equal(fmax.cpu().numpy().view(np.uint32), u["exp_max"].view(np.uint32)), n
        assert np.array_equal(moved.cpu().numpy(), u["exp_moved"]), n


@pytest.mark.parametrize("api", ["host", "device"])
def test_gpu_pairs_match_reference(ctx, fixture, api):
    for n in dynio.cases(fixture):
        p = bpio.pairs_case(dynio.capture(fixture, n))
        m = len(p["body"])
        for axis in (-1, 0, 1, 2):
            if api == "host":
                bp = BP.make(m, 0, 0, body=p["body"], category=p["category"], mask=p["mask"], fat_min=p["fat_min"],
                             fat_max=p["fat_max"])
                cnt, pairs = ctx.broadphase_pairs(bp, 4096, axis=axis)
            else:
                keep = [T(p[k]) for k in ("body", "category", "mask", "fat_min", "fat_max")]
                bp = BP.make(m, 0, 0, body=keep[0], category=keep[1], mask=keep[2], fat_min=keep[3], fat_max=keep[4])
                c, pr = ctx.broadphase_pairs(bp, 4096, axis=axis, device=True)
                ctx.synchronize()
                cnt, pairs = int(c.item()), pr.cpu().numpy()
            assert cnt == len(p["expected"]), (n, axis)
            assert bpio.pair_set(pairs, cnt, p["index"]) == p["expected"], (n, axis)


@pytest.mark.parametrize("seed,n,groups", [(1, 20000, 0), (2, 50000, 37), (3, 3000, 0)])
def test_gpu_pairs_random_vs_oracle(ctx, port, seed, n, groups):
    """Random AABBs (one world, or 37 worlds), a body shared by some colliders
    and filter bits, every sweep axis, against the brute-force oracle."""
    rng = np.random.default_rng(seed)
    mn, mx, body, grp = bpio.random_aabbs(n, rng, world=60.0 if n > 10000 else 15.0, groups=groups,
                                          nbodies=int(n * 0.9))
    cat = (1 << rng.integers(0, 3, n)).astype(np.uint16)
    msk = np.where(rng.random(n) < 0.2, 0xffff & ~2, 0xffff).astype(np.uint16)
    if groups:
        exp = set()
        for g in range(groups):
            idx = np.flatnonzero(grp == g)
            e = bpio.oracle_pairs(port.lib, mn[idx], mx[idx], body[idx], None, cat[idx], msk[idx])
            exp |= bpio.pair_set(e, len(e), idx)
    else:
        e = bpio.oracle_pairs(port.lib, mn, mx, body, None, cat, msk)
        exp = bpio.pair_set(e, len(e))
    keep = [T(a) for a in (body, cat, msk, mn, mx)] + ([T(grp)] if groups else [None])
    bp = BP.make(n, 0, groups, body=keep[0], category=keep[1], mask=keep[2], fat_min=keep[3], fat_max=keep[4],
                 group=keep[5])
    for axis in (-1, 0, 1, 2):
        c, pr = ctx.broadphase_pairs(bp, len(exp) + 16, axis=axis, device=True)
        ctx.synchronize()
        cnt = int(c.item())
        assert cnt == len(exp)
        got = pr.cpu().numpy()[:cnt]
        assert np.all(got[:, 0] < got[:, 1])
        assert bpio.pair_set(got, cnt) == exp
    assert ctx.device_errors(clear=True) & 8 == 0


def test_gpu_pairs_many_worlds(ctx, fixture):
    """4,096 worlds (the fixture worlds repeated) as groups of one call: the
    pairs are each world's reference pairs, remapped."""
    cases = [bpio.pairs_case(dynio.capture(fixture, n)) for n in dynio.cases(fixture)]
    worlds = (cases * (4096 // len(cases) + 1))[:4096]
    cols = {k: [] for k in ("body", "category", "mask", "fat_min", "fat_max")}
    group, expected, off, boff = [], set(), 0, 0
    for g, w in enumerate(worlds):
        m = len(w["body"])
        for k in cols:
            cols[k].append(w[k] + (boff if k == "body" else 0))
        group.append(np.full(m, g, np.int32))
        pos = {int(c): off + j for j, c in enumerate(w["index"])}
        expected |= {(pos[a], pos[b]) for a, b in w["expected"]}
        off += m
        boff += int(w["body"].max()) + 1
    arr = {k: np.concatenate(v) for k, v in cols.items()}
    keep = [T(arr[k]) for k in ("body", "category", "mask", "fat_min", "fat_max")] + [T(np.concatenate(group))]
    bp = BP.make(off, 0, 4096, body=keep[0], category=keep[1], mask=keep[2], fat_min=keep[3], fat_max=keep[4],
                 group=keep[5])
    for axis in (-1, 0):
        c, pr = ctx.broadphase_pairs(bp, len(expected) + 16, axis=axis, device=True)
        ctx.synchronize()
        cnt = int(c.item())
        assert cnt == len(expected)
        assert bpio.pair_set(pr.cpu().numpy(), cnt) == expected


def test_gpu_broadphase_errors(ctx):
    z = np.zeros((1, 4), np.float32)
    bp = BP.make(1, 0, 0, body=np.zeros(1, np.int32), fat_min=z, fat_max=z)
    with pytest.raises(engine.Rp3dgError):
        ctx.broadphase_pairs(bp, 4, axis=3)
    with pytest.raises(engine.Rp3dgError):
        ctx.broadphase_pairs(bp, 4, axis=-2)
    for axis in (-1, 0):
        cnt, _ = ctx.broadphase_pairs(BP.make(0, 0, 0), 4, axis=axis)
        assert cnt == 0
        cnt, _ = ctx.broadphase_pairs(bp, 4, axis=axis)   # one collider: no pair
        assert cnt == 0
