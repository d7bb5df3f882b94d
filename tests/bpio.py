"""Broad-phase inputs and expected outputs from a reference capture
(tests/golden/np_dynamics.npz or reflib.RefWorld.capture)."""
import ctypes as C

import numpy as np

from reactphysics3d_b200 import _abi as A


def shapes(cap):
    """A shape table with one entry per collider (rp3dg.h kinds)."""
    n = len(cap["bp_id"])
    t = np.zeros(n, A.SHAPE_DTYPE)
    t["kind"] = cap["bp_shape"][:, 3].astype(np.int32)
    t["params"][:, :3] = cap["bp_shape"][:, :3]
    return t


def update_case(cap):
    """Colliders the reference updated at the end of the step (enabled, in the
    broad phase): their indices, shape ids, world transforms, fat AABBs before,
    and the expected fat AABBs and moved flags after."""
    nce = int(cap["in_collider_nb_enabled"][0])
    upd = np.flatnonzero((cap["bp_id"] >= 0)[:nce])
    c = lambda a: np.ascontiguousarray(a[upd])
    # reinserted = the fat AABB changed (a reinsertion always changes it); the
    # reference's moved set also holds colliders of bodies woken during the
    # step (RigidBody::setIsSleeping -> askForBroadPhaseCollisionCheck),
    # which are not reinserted
    fin = np.concatenate([cap["bp_in_fat_min"], cap["bp_in_fat_max"]], 1).view(np.uint32)
    fout = np.concatenate([cap["bp_out_fat_min"], cap["bp_out_fat_max"]], 1).view(np.uint32)
    reinserted = np.any(fin != fout, axis=1).astype(np.uint8)
    assert np.all(cap["bp_moved"][reinserted == 1] == 1)
    return {"index": upd, "shape": upd.astype(np.int32), "wpos": c(cap["out_collider_world_position"]),
            "wori": c(cap["out_collider_world_orientation"]), "fat_min": c(cap["bp_in_fat_min"]),
            "fat_max": c(cap["bp_in_fat_max"]), "exp_min": c(cap["bp_out_fat_min"]),
            "exp_max": c(cap["bp_out_fat_max"]), "exp_moved": c(reinserted)}


def pairs_case(cap):
    """Colliders in the broad phase at the start of the step with their fat
    AABBs, bodies and filter bits, and the reference's pair set after the
    step's broad phase (collider indices)."""
    inb = np.flatnonzero(cap["bp_id"] >= 0)
    c = lambda a: np.ascontiguousarray(a[inb])
    return {"index": inb, "fat_min": c(cap["bp_start_fat_min"]), "fat_max": c(cap["bp_start_fat_max"]),
            "body": c(cap["in_collider_body"]).astype(np.int32),
            "category": c(cap["bp_bits"][:, 0]).astype(np.uint16), "mask": c(cap["bp_bits"][:, 1]).astype(np.uint16),
            "expected": set(map(tuple, cap["bp_pairs"].tolist()))}


def pair_set(pairs, count, index=None):
    p = np.asarray(pairs)[:count]
    if index is not None:
        p = np.sort(index[p], axis=1)
    return set(map(tuple, p.tolist()))


def bind_oracle(lib):
    lib.rp3do_broadphase_update.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rp3do_broadphase_pairs.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_long]
    lib.rp3do_broadphase_pairs.restype = C.c_long


def oracle_update(lib, table, case):
    bind_oracle(lib)
    fmin, fmax = case["fat_min"].copy(), case["fat_max"].copy()
    moved = np.zeros(len(fmin), np.uint8)
    lib.rp3do_broadphase_update(table.ctypes.data, None, len(fmin), case["shape"].ctypes.data, case["wpos"].ctypes.data,
                                case["wori"].ctypes.data, None, fmin.ctypes.data, fmax.ctypes.data, moved.ctypes.data)
    return fmin, fmax, moved


def oracle_pairs(lib, fat_min, fat_max, body, group=None, category=None, mask=None, cap=1 << 22):
    bind_oracle(lib)
    out = np.zeros((cap, 2), np.int32)
    p = lambda a: None if a is None else np.ascontiguousarray(a).ctypes.data
    n = lib.rp3do_broadphase_pairs(len(fat_min), p(fat_min), p(fat_max), p(body), p(group), p(category), p(mask),
                                   out.ctypes.data, cap)
    assert n <= cap
    return out[:n]


def random_aabbs(n, rng, world=20.0, size=(0.2, 1.5), groups=0, nbodies=None):
    c = rng.uniform(-world, world, (n, 3)).astype(np.float32)
    h = rng.uniform(size[0], size[1], (n, 3)).astype(np.float32)
    mn = np.zeros((n, 4), np.float32); mx = np.zeros((n, 4), np.float32)
    mn[:, :3] = c - h; mx[:, :3] = c + h
    body = (rng.integers(0, nbodies, n) if nbodies else np.arange(n)).astype(np.int32)
    grp = np.sort(rng.integers(0, groups, n)).astype(np.int32) if groups else None
    return mn, mx, body, grp
