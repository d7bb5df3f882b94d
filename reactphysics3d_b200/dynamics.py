"""Dynamics stage of a world step through the C ABI (include/rp3dg.h,
rp3dg_dynamics_step_host / rp3dg_dynamics_step_device).

`DynWorld` holds one world's dynamics-stage state as numpy arrays (host) or
torch CUDA tensors (device), named after the reference's component arrays
(RigidBodyComponents, ColliderComponents, ContactManifold, ContactPoint,
Islands).  `structs()` returns the ctypes structures the library takes.
"""
import ctypes as C

import numpy as np

BODY_F4 = ("position", "orientation", "com_world", "com_local", "linear_velocity", "angular_velocity", "force",
           "torque", "inv_inertia_local", "mass", "linear_lock", "angular_lock")
BODY_FIELDS = BODY_F4 + ("inv_inertia_world", "gravity")
COLLIDER_FIELDS = ("body", "local_position", "local_orientation", "world_position", "world_orientation", "material")
MANIFOLD_FIELDS = ("ids", "point_start", "nb_points", "friction_vector1", "friction_vector2", "friction_impulse")
POINT_FIELDS = ("normal_depth", "local1", "local2", "penetration_impulse", "is_resting")
ISLAND_FIELDS = ("manifold_start", "manifold_count")
# arrays the stage writes
OUTPUTS = ("position", "orientation", "com_world", "linear_velocity", "angular_velocity", "inv_inertia_world",
           "world_position", "world_orientation", "friction_vector1", "friction_vector2", "friction_impulse",
           "penetration_impulse", "is_resting")

DTYPES = {"gravity": np.uint8, "body": np.int32, "ids": np.int32, "point_start": np.uint32, "nb_points": np.uint8,
          "penetration_impulse": np.float32, "is_resting": np.uint8, "manifold_start": np.uint32,
          "manifold_count": np.uint32}


class Bodies(C.Structure):
    _fields_ = [("n", C.c_uint32), ("n_enabled", C.c_uint32)] + [(f, C.c_void_p) for f in (
        "position", "orientation", "com_world", "com_local", "linear_velocity", "angular_velocity", "force", "torque",
        "inv_inertia_local", "inv_inertia_world", "mass", "linear_lock", "angular_lock", "gravity")]


class Colliders(C.Structure):
    _fields_ = [("n", C.c_uint32), ("n_enabled", C.c_uint32)] + [(f, C.c_void_p) for f in COLLIDER_FIELDS]


class Manifolds(C.Structure):
    _fields_ = [("n", C.c_uint32)] + [(f, C.c_void_p) for f in MANIFOLD_FIELDS]


class Points(C.Structure):
    _fields_ = [("n", C.c_uint32)] + [(f, C.c_void_p) for f in POINT_FIELDS]


class Islands(C.Structure):
    _fields_ = [("n", C.c_uint32)] + [(f, C.c_void_p) for f in ISLAND_FIELDS]


class Params(C.Structure):
    _fields_ = [("dt", C.c_float), ("gravity", C.c_float * 3), ("gravity_enabled", C.c_int32),
                ("velocity_iterations", C.c_int32), ("split_impulse", C.c_int32),
                ("restitution_velocity_threshold", C.c_float)]


def make_params(dt=1.0 / 60.0, gravity=(0.0, -9.81, 0.0), gravity_enabled=True, iterations=6, split=True,
                restitution_threshold=0.5):
    """WorldSettings defaults (PhysicsWorld.h:120-135)."""
    return Params(float(dt), (C.c_float * 3)(*map(float, gravity)), int(gravity_enabled), int(iterations), int(split),
                  float(restitution_threshold))


class DynWorld:
    """Dynamics-stage arrays of one or more worlds (bodies, colliders,
    manifolds in solver order, points, islands as manifold ranges)."""

    def __init__(self, arrays, nb_enabled, nc_enabled, device=None):
        self.a = {}
        for k, v in arrays.items():
            v = np.ascontiguousarray(v, dtype=DTYPES.get(k, np.float32))
            if device is not None:
                import torch
                v = torch.from_numpy(v.copy()).to(device)
            self.a[k] = v
        self.device = device
        self.nb_enabled, self.nc_enabled = int(nb_enabled), int(nc_enabled)

    def __getitem__(self, k):
        return self.a[k]

    def _n(self, k):
        return int(self.a[k].shape[0])

    def _p(self, k):
        v = self.a[k]
        if self._n(k) == 0:
            return None
        return v.data_ptr() if self.device is not None else v.ctypes.data

    def structs(self):
        b = Bodies(self._n("mass"), self.nb_enabled, *[self._p(f) for f in (
            "position", "orientation", "com_world", "com_local", "linear_velocity", "angular_velocity", "force",
            "torque", "inv_inertia_local", "inv_inertia_world", "mass", "linear_lock", "angular_lock", "gravity")])
        c = Colliders(self._n("body"), self.nc_enabled, *[self._p(f) for f in COLLIDER_FIELDS])
        m = Manifolds(self._n("ids"), *[self._p(f) for f in MANIFOLD_FIELDS])
        p = Points(self._n("normal_depth"), *[self._p(f) for f in POINT_FIELDS])
        i = Islands(self._n("manifold_start"), *[self._p(f) for f in ISLAND_FIELDS])
        return b, c, m, p, i

    def host(self):
        """A host copy (numpy) of a device world."""
        if self.device is None:
            return self
        return DynWorld({k: v.cpu().numpy() for k, v in self.a.items()}, self.nb_enabled, self.nc_enabled)

    def copy(self):
        h = self.host()
        return DynWorld({k: np.array(v, copy=True) for k, v in h.a.items()}, self.nb_enabled, self.nc_enabled)

    @property
    def counts(self):
        return {"bodies": self._n("mass"), "colliders": self._n("body"), "manifolds": self._n("ids"),
                "points": self._n("normal_depth"), "islands": self._n("manifold_start")}


def bind(lib, fn):
    getattr(lib, fn).argtypes = [C.POINTER(Params), C.POINTER(Bodies), C.POINTER(Colliders), C.POINTER(Manifolds),
                                 C.POINTER(Points), C.POINTER(Islands)]


def world_from_capture(cap, prefix="in_"):
    """DynWorld from a reference capture (tests/reflib.RefWorld.capture)."""
    g = lambda k: cap[prefix + k]
    arrays = {
        "position": g("body_position"), "orientation": g("body_orientation"), "com_world": g("body_com_world"),
        "com_local": g("body_com_local"), "linear_velocity": g("body_linear_velocity"),
        "angular_velocity": g("body_angular_velocity"), "force": g("body_force"), "torque": g("body_torque"),
        "inv_inertia_local": g("body_inv_inertia_local"), "mass": g("body_mass"),
        "linear_lock": g("body_linear_lock"), "angular_lock": g("body_angular_lock"), "gravity": g("body_gravity"),
        "inv_inertia_world": g("body_inv_inertia_world").reshape(-1, 4),
        "body": g("collider_body"), "local_position": g("collider_local_position"),
        "local_orientation": g("collider_local_orientation"), "world_position": g("collider_world_position"),
        "world_orientation": g("collider_world_orientation"), "material": g("collider_material"),
        "ids": g("manifold_ids").reshape(-1, 4), "point_start": g("manifold_point_start"),
        "nb_points": g("manifold_nb_points"), "friction_vector1": g("manifold_friction_vector1"),
        "friction_vector2": g("manifold_friction_vector2"), "friction_impulse": g("manifold_friction_impulse"),
        "normal_depth": g("point_normal_depth"), "local1": g("point_local1"), "local2": g("point_local2"),
        "penetration_impulse": g("point_penetration_impulse"), "is_resting": g("point_is_resting"),
        "manifold_start": g("island_manifold_start"), "manifold_count": g("island_manifold_count"),
    }
    return DynWorld(arrays, int(g("body_nb_enabled")[0]), int(g("collider_nb_enabled")[0]))


def params_from_capture(cap):
    p = cap["params"]
    return make_params(dt=p[0], gravity=p[1:4], gravity_enabled=p[4] != 0, iterations=int(p[5]), split=p[6] != 0,
                       restitution_threshold=p[7])


def batch_worlds(worlds):
    """Concatenate independent worlds into one DynWorld (one launch for all).

    Enabled bodies (and colliders) of every world come first, in world order,
    then the read-only ones; body, collider, point and manifold indices are
    remapped.  Returns (batched world, layout) where layout lets
    `unbatch_worlds` split the result back."""
    nb = [w._n("mass") for w in worlds]
    nc = [w._n("body") for w in worlds]
    ne_b = [w.nb_enabled for w in worlds]
    ne_c = [w.nc_enabled for w in worlds]
    tot_eb, tot_ec = sum(ne_b), sum(ne_c)
    body_map, coll_map = [], []
    eb = ob = ec = oc = 0
    for k, w in enumerate(worlds):
        m = np.empty(nb[k], np.int64)
        m[: ne_b[k]] = np.arange(eb, eb + ne_b[k])
        m[ne_b[k]:] = np.arange(tot_eb + ob, tot_eb + ob + nb[k] - ne_b[k])
        eb += ne_b[k]; ob += nb[k] - ne_b[k]
        body_map.append(m)
        c = np.empty(nc[k], np.int64)
        c[: ne_c[k]] = np.arange(ec, ec + ne_c[k])
        c[ne_c[k]:] = np.arange(tot_ec + oc, tot_ec + oc + nc[k] - ne_c[k])
        ec += ne_c[k]; oc += nc[k] - ne_c[k]
        coll_map.append(c)
    NB, NC = sum(nb), sum(nc)
    out = {}
    for f in BODY_F4 + ("gravity",):
        a0 = worlds[0].host()[f]
        arr = np.zeros((NB,) + a0.shape[1:], a0.dtype)
        for k, w in enumerate(worlds):
            arr[body_map[k]] = w.host()[f]
        out[f] = arr
    iiw = np.zeros((NB, 3, 4), np.float32)
    for k, w in enumerate(worlds):
        iiw[body_map[k]] = np.asarray(w.host()["inv_inertia_world"]).reshape(-1, 3, 4)
    out["inv_inertia_world"] = iiw.reshape(-1, 4)
    for f in COLLIDER_FIELDS:
        a0 = worlds[0].host()[f]
        arr = np.zeros((NC,) + a0.shape[1:], a0.dtype)
        for k, w in enumerate(worlds):
            v = np.array(w.host()[f])
            if f == "body":
                v = body_map[k][v].astype(np.int32)
            arr[coll_map[k]] = v
        out[f] = arr
    mans = {f: [] for f in MANIFOLD_FIELDS}
    pts = {f: [] for f in POINT_FIELDS}
    isl = {f: [] for f in ISLAND_FIELDS}
    m_off = p_off = 0
    layout = []
    for k, w in enumerate(worlds):
        h = w.host()
        ids = np.array(h["ids"]).reshape(-1, 4).astype(np.int64)
        ids[:, 0] = body_map[k][ids[:, 0]]; ids[:, 1] = body_map[k][ids[:, 1]]
        ids[:, 2] = coll_map[k][ids[:, 2]]; ids[:, 3] = coll_map[k][ids[:, 3]]
        mans["ids"].append(ids.astype(np.int32))
        mans["point_start"].append(np.asarray(h["point_start"]) + p_off)
        for f in ("nb_points", "friction_vector1", "friction_vector2", "friction_impulse"):
            mans[f].append(np.asarray(h[f]))
        for f in POINT_FIELDS:
            pts[f].append(np.asarray(h[f]))
        isl["manifold_start"].append(np.asarray(h["manifold_start"]) + m_off)
        isl["manifold_count"].append(np.asarray(h["manifold_count"]))
        nm_k, np_k = len(ids), len(np.asarray(h["normal_depth"]))
        layout.append((body_map[k], coll_map[k], m_off, nm_k, p_off, np_k, ne_b[k], ne_c[k]))
        m_off += nm_k
        p_off += np_k
    for d in (mans, pts, isl):
        for f, v in d.items():
            out[f] = np.concatenate(v) if v else np.zeros(0)
    return DynWorld(out, tot_eb, tot_ec), layout


def unbatch_worlds(world, layout):
    """Split a batched world back into its worlds (host copies)."""
    h = world.host()
    res = []
    for bm, cm, m0, nm, p0, npt, neb, nec in layout:
        a = {}
        for f in BODY_F4 + ("gravity",):
            a[f] = np.asarray(h[f])[bm]
        a["inv_inertia_world"] = np.asarray(h["inv_inertia_world"]).reshape(-1, 3, 4)[bm].reshape(-1, 4)
        for f in COLLIDER_FIELDS:
            a[f] = np.asarray(h[f])[cm]
        for f in MANIFOLD_FIELDS:
            a[f] = np.asarray(h[f])[m0:m0 + nm]
        for f in POINT_FIELDS:
            a[f] = np.asarray(h[f])[p0:p0 + npt]
        a["manifold_start"] = np.zeros(0, np.uint32)
        a["manifold_count"] = np.zeros(0, np.uint32)
        res.append(DynWorld(a, neb, nec))
    return res
