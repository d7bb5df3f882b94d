"""Dynamics-stage fixtures (tests/golden/np_dynamics.npz) and comparisons."""
import ctypes as C

import numpy as np

from reactphysics3d_b200 import dynamics as D

# output array of the stage -> (captured field, rows compared: "b" enabled
# bodies, "c" enabled colliders, None all)
OUT_CHECKS = {
    "position": ("out_body_position", "b"), "orientation": ("out_body_orientation", "b"),
    "com_world": ("out_body_com_world", "b"), "linear_velocity": ("out_body_linear_velocity", "b"),
    "angular_velocity": ("out_body_angular_velocity", "b"),
    "world_position": ("out_collider_world_position", "c"),
    "world_orientation": ("out_collider_world_orientation", "c"),
    "friction_vector1": ("out_manifold_friction_vector1", None),
    "friction_vector2": ("out_manifold_friction_vector2", None),
    "friction_impulse": ("out_manifold_friction_impulse", None),
    "penetration_impulse": ("out_point_penetration_impulse", None),
    "is_resting": ("out_point_is_resting", None),
}


def cases(z):
    return sorted({k.split("/")[0] for k in z.files})


def capture(z, name):
    pre = name + "/"
    return {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}


def mismatches(world, cap):
    """{array: number of rows differing in any bit} against the reference."""
    h = world.host()
    lim = {"b": h.nb_enabled, "c": h.nc_enabled, None: None}
    bad = {}
    for k, (ck, rows) in OUT_CHECKS.items():
        a, b = np.asarray(h[k]), cap[ck]
        n = lim[rows]
        if n is not None:
            a, b = a[:n], b[:n]
        if a.dtype == np.float32:
            a, b = a.view(np.uint32), b.view(np.uint32)
        if len(a) and len(a) == len(b):
            nbad = int(np.sum(np.any((a != b).reshape(len(a), -1), axis=1)))
        else:
            nbad = 0 if len(a) == len(b) else -1
        if nbad:
            bad[k] = nbad
    ne = h.nb_enabled
    iiw = np.asarray(h["inv_inertia_world"]).reshape(-1, 3, 4)[:ne]
    if not np.array_equal(iiw.view(np.uint32), cap["out_body_inv_inertia_world"][:ne].view(np.uint32)):
        bad["inv_inertia_world"] = 1
    return bad


def run_oracle(lib, params, world):
    D.bind(lib, "rp3do_dynamics_step")
    b, c, m, p, i = world.structs()
    rc = lib.rp3do_dynamics_step(C.byref(params), C.byref(b), C.byref(c), C.byref(m), C.byref(p), C.byref(i))
    assert rc == 0, rc
    return world
