"""Broad phase through the C ABI (include/rp3dg.h: rp3dg_broadphase_update_device,
rp3dg_broadphase_pairs_device / _host): collider fat AABBs and the set of
overlapping pairs."""
import ctypes as C

import numpy as np


class BroadPhase(C.Structure):
    _fields_ = [("n", C.c_uint32), ("n_update", C.c_uint32), ("nb_groups", C.c_uint32)] + [
        (f, C.c_void_p) for f in ("shape", "body", "group", "category", "mask", "world_position",
                                  "world_orientation", "force_reinsert", "fat_min", "fat_max", "moved")]


def bind(lib):
    P = C.c_void_p
    lib.rp3dg_broadphase_update_device.argtypes = [P, C.POINTER(BroadPhase)]
    for fn in ("rp3dg_broadphase_pairs_device", "rp3dg_broadphase_pairs_host"):
        getattr(lib, fn).argtypes = [P, C.POINTER(BroadPhase), C.c_int, P, C.c_uint32, P]


def _ptr(a):
    if a is None:
        return None
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


def make(n, n_update=0, nb_groups=0, shape=None, body=None, group=None, category=None, mask=None,
         world_position=None, world_orientation=None, force_reinsert=None, fat_min=None, fat_max=None, moved=None):
    """The ctypes structure over numpy arrays (host call) or torch CUDA
    tensors (device calls); the arrays must stay alive during the call."""
    return BroadPhase(n, n_update, nb_groups, _ptr(shape), _ptr(body), _ptr(group), _ptr(category), _ptr(mask),
                      _ptr(world_position), _ptr(world_orientation), _ptr(force_reinsert), _ptr(fat_min),
                      _ptr(fat_max), _ptr(moved))
