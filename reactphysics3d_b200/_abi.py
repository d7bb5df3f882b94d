"""ctypes mirror of the C ABI in include/rp3dg.h.

The structs here are byte-for-byte the ones the CUDA library exports; the
numpy helpers build struct-of-arrays pair batches and contact buffers and hand
their data pointers to the library.  Both the library (`librp3dg.so`) and any
other shared object exporting the same layout can be driven through them.
"""
import ctypes as C

import numpy as np

MAX_CONTACTS = 16  # NB_MAX_CONTACT_POINTS_IN_NARROWPHASE_INFO (configuration.h:109)

SHAPE_SPHERE, SHAPE_CAPSULE, SHAPE_BOX, SHAPE_CONVEX_MESH, SHAPE_HEIGHTFIELD, SHAPE_CONCAVE_MESH = 0, 1, 2, 3, 4, 5

ALGO_NONE = 0
ALGO_SPHERE_VS_SPHERE = 1
ALGO_SPHERE_VS_CAPSULE = 2
ALGO_CAPSULE_VS_CAPSULE = 3
ALGO_SPHERE_VS_CONVEX_POLYHEDRON = 4
ALGO_CAPSULE_VS_CONVEX_POLYHEDRON = 5
ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON = 6

LF_IS_VALID = 0x01
LF_WAS_COLLIDING = 0x02
LF_WAS_USING_GJK = 0x04
LF_WAS_USING_SAT = 0x08
LF_SAT_FACE_POLY1 = 0x10
LF_SAT_FACE_POLY2 = 0x20
LF_IS_OBSOLETE = 0x40

SHAPE_DTYPE = np.dtype([("params", "<f4", (4,)), ("kind", "<i4"), ("mesh", "<i4"), ("reserved", "<i4", (2,))])
CACHE_DTYPE = np.dtype([("gjk_axis", "<f4", (3,)), ("flags", "u1"), ("sat_face", "u1"),
                        ("sat_edge1", "u1"), ("sat_edge2", "u1")])
assert SHAPE_DTYPE.itemsize == 32 and CACHE_DTYPE.itemsize == 16


class PairBatch(C.Structure):
    _fields_ = [("n", C.c_uint32),
                ("shape1", C.c_void_p), ("shape2", C.c_void_p),
                ("pos1", C.c_void_p), ("rot1", C.c_void_p),
                ("pos2", C.c_void_p), ("rot2", C.c_void_p),
                ("report_contacts", C.c_void_p), ("cache", C.c_void_p)]


class ContactBatch(C.Structure):
    _fields_ = [("is_colliding", C.c_void_p), ("nb_contacts", C.c_void_p),
                ("normal_depth", C.c_void_p), ("local1", C.c_void_p), ("local2", C.c_void_p),
                ("max_contacts", C.c_uint32)]


def fresh_cache(n):
    """LastFrameCollisionInfo() defaults (OverlappingPairs.h:86-91)."""
    c = np.zeros(n, dtype=CACHE_DTYPE)
    c["gjk_axis"][:, 1] = 1.0
    return c


def _ptr(a):
    return None if a is None else a.ctypes.data


class HostPairs:
    """A pair batch held in numpy arrays (host memory)."""

    def __init__(self, shape1, shape2, pos1, rot1, pos2, rot2, report=None, cache=None):
        self.shape1 = np.ascontiguousarray(shape1, dtype=np.int32)
        self.shape2 = np.ascontiguousarray(shape2, dtype=np.int32)
        self.pos1 = np.ascontiguousarray(pos1, dtype=np.float32).reshape(-1, 4)
        self.rot1 = np.ascontiguousarray(rot1, dtype=np.float32).reshape(-1, 4)
        self.pos2 = np.ascontiguousarray(pos2, dtype=np.float32).reshape(-1, 4)
        self.rot2 = np.ascontiguousarray(rot2, dtype=np.float32).reshape(-1, 4)
        self.report = None if report is None else np.ascontiguousarray(report, dtype=np.uint8)
        self.cache = None if cache is None else np.ascontiguousarray(cache, dtype=CACHE_DTYPE)

    @property
    def n(self):
        return int(self.shape1.shape[0])

    def slice(self, begin, end):
        return HostPairs(self.shape1[begin:end], self.shape2[begin:end], self.pos1[begin:end],
                         self.rot1[begin:end], self.pos2[begin:end], self.rot2[begin:end],
                         None if self.report is None else self.report[begin:end],
                         None if self.cache is None else self.cache[begin:end].copy())

    def struct(self):
        return PairBatch(self.n, _ptr(self.shape1), _ptr(self.shape2), _ptr(self.pos1), _ptr(self.rot1),
                         _ptr(self.pos2), _ptr(self.rot2), _ptr(self.report), _ptr(self.cache))


class HostContacts:
    """Per-pair narrow-phase results in host memory (slot-major contacts)."""

    def __init__(self, n, max_contacts=MAX_CONTACTS):
        self.n = n
        self.max_contacts = max_contacts
        self.is_colliding = np.zeros(n, dtype=np.uint8)
        self.nb_contacts = np.zeros(n, dtype=np.uint8)
        self.normal_depth = np.zeros((max_contacts, n, 4), dtype=np.float32)
        self.local1 = np.zeros((max_contacts, n, 4), dtype=np.float32)
        self.local2 = np.zeros((max_contacts, n, 4), dtype=np.float32)

    def struct(self):
        return ContactBatch(_ptr(self.is_colliding), _ptr(self.nb_contacts), _ptr(self.normal_depth),
                            _ptr(self.local1), _ptr(self.local2), self.max_contacts)

    def valid_mask(self):
        """Boolean [max_contacts, n] mask of the slots that hold a contact."""
        return np.arange(self.max_contacts)[:, None] < self.nb_contacts[None, :]


# ---- world step (rp3dg_world_*) --------------------------------------------
BODY_STATIC, BODY_KINEMATIC, BODY_DYNAMIC = 0, 1, 2

WORLD_SETTINGS_DTYPE = np.dtype([
    ("gravity", "<f4", (3,)), ("velocity_iterations", "<i4"), ("sleeping_enabled", "<i4"),
    ("sleep_linear_velocity", "<f4"), ("sleep_angular_velocity", "<f4"), ("time_before_sleep", "<f4"),
    ("restitution_velocity_threshold", "<f4"), ("persistent_contact_distance_threshold", "<f4"),
    ("cos_angle_similar_contact_manifold", "<f4"), ("position_iterations", "<i4")])
BODY_DESC_DTYPE = np.dtype([
    ("type", "<i4"), ("position", "<f4", (3,)), ("orientation", "<f4", (4,)),
    ("linear_velocity", "<f4", (3,)), ("angular_velocity", "<f4", (3,)),
    ("linear_damping", "<f4"), ("angular_damping", "<f4"),
    ("linear_lock", "<f4", (3,)), ("angular_lock", "<f4", (3,)),
    ("gravity_enabled", "<i4"), ("allowed_to_sleep", "<i4")])
COLLIDER_DESC_DTYPE = np.dtype([
    ("body", "<i4"), ("shape", "<i4"), ("position", "<f4", (3,)), ("orientation", "<f4", (4,)),
    ("friction", "<f4"), ("bounciness", "<f4"), ("mass_density", "<f4"),
    ("category", "<u2"), ("mask", "<u2"), ("flags", "<u4")])
COLLIDER_TRIGGER = 1
WORLD_STATS_DTYPE = np.dtype([(k, "<u4") for k in (
    "overlapping_pairs", "disabled_pairs", "narrowphase_tests", "contact_pairs", "manifolds",
    "contact_points", "islands", "enabled_bodies", "moved_colliders", "reserved")])
JOINT_BALL_AND_SOCKET, JOINT_HINGE, JOINT_FIXED, JOINT_SLIDER = 0, 1, 2, 3
JOINT_DESC_DTYPE = np.dtype([
    ("type", "<i4"), ("body1", "<i4"), ("body2", "<i4"), ("anchor", "<f4", (3,)), ("axis", "<f4", (3,)),
    ("collision_enabled", "<i4"), ("cone_limit_enabled", "<i4"), ("cone_half_angle", "<f4"),
    ("limit_enabled", "<i4"), ("min_angle", "<f4"), ("max_angle", "<f4"),
    ("motor_enabled", "<i4"), ("motor_speed", "<f4"), ("max_motor_torque", "<f4")])
assert JOINT_DESC_DTYPE.itemsize == 72
CONTACT_START, CONTACT_STAY, CONTACT_EXIT = 0, 1, 2
CONTACT_EVENT_DTYPE = np.dtype([("body1", "<i4"), ("body2", "<i4"), ("collider1", "<i4"), ("collider2", "<i4"),
                                ("type", "<i4"), ("first_point", "<u4"), ("nb_points", "<u4")])
assert CONTACT_EVENT_DTYPE.itemsize == 28
RAYCAST_CLOSEST, RAYCAST_ANY, RAYCAST_ALL = 0, 1, 2
RAY_DTYPE = np.dtype([("point1", "<f4", (3,)), ("point2", "<f4", (3,)), ("max_fraction", "<f4"),
                      ("category_mask", "<u4")])
RAYCAST_HIT_DTYPE = np.dtype([("world_point", "<f4", (3,)), ("world_normal", "<f4", (3,)), ("hit_fraction", "<f4"),
                              ("body", "<i4"), ("collider", "<i4"), ("flags", "<i4")])
assert RAY_DTYPE.itemsize == 32 and RAYCAST_HIT_DTYPE.itemsize == 40
# DebugRenderer::DebugItem bits and DebugLine / DebugTriangle
DEBUG_COLLIDER_AABB, DEBUG_COLLIDER_BROADPHASE_AABB, DEBUG_COLLISION_SHAPE = 0x01, 0x02, 0x04
DEBUG_CONTACT_POINT, DEBUG_CONTACT_NORMAL, DEBUG_COLLISION_SHAPE_NORMAL = 0x08, 0x10, 0x20
DEBUG_ALL = 0x3f
DEBUG_LINE_DTYPE = np.dtype([("p1", "<f4", (3,)), ("color1", "<u4"), ("p2", "<f4", (3,)), ("color2", "<u4")])
DEBUG_TRIANGLE_DTYPE = np.dtype([("p1", "<f4", (3,)), ("color1", "<u4"), ("p2", "<f4", (3,)), ("color2", "<u4"),
                                 ("p3", "<f4", (3,)), ("color3", "<u4")])
assert DEBUG_LINE_DTYPE.itemsize == 32 and DEBUG_TRIANGLE_DTYPE.itemsize == 48
assert WORLD_SETTINGS_DTYPE.itemsize == 48 and BODY_DESC_DTYPE.itemsize == 96
assert COLLIDER_DESC_DTYPE.itemsize == 56 and WORLD_STATS_DTYPE.itemsize == 40


def default_world_settings():
    """PhysicsWorld::WorldSettings defaults (PhysicsWorld.h:122-138), float32."""
    s = np.zeros(1, WORLD_SETTINGS_DTYPE)[0]
    f = np.float32
    s["gravity"] = (0.0, -9.81, 0.0)
    s["velocity_iterations"] = 6
    s["sleeping_enabled"] = 1
    s["sleep_linear_velocity"] = f(0.02)
    s["sleep_angular_velocity"] = f(3.0) * (f(3.141592653589) / f(180.0))
    s["time_before_sleep"] = 1.0
    s["restitution_velocity_threshold"] = f(0.5)
    s["persistent_contact_distance_threshold"] = f(0.03)
    s["cos_angle_similar_contact_manifold"] = f(0.95)
    s["position_iterations"] = 3
    return s


def rays(n):
    """Ray defaults: maxFraction 1, category mask 0xFFFF."""
    r = np.zeros(n, RAY_DTYPE)
    r["max_fraction"] = 1.0
    r["category_mask"] = 0xFFFF
    return r


def joint_descs(n):
    """JointInfo defaults: collision enabled, no cone limit (half angle PI),
    hinge / slider limits off (-1, 1), no motor."""
    j = np.zeros(n, JOINT_DESC_DTYPE)
    j["collision_enabled"] = 1
    j["cone_half_angle"] = np.float32(3.141592653589)
    j["min_angle"] = -1.0
    j["max_angle"] = 1.0
    return j


def body_descs(n):
    b = np.zeros(n, BODY_DESC_DTYPE)
    b["type"] = BODY_DYNAMIC
    b["orientation"][:, 3] = 1.0
    b["linear_lock"] = 1.0
    b["angular_lock"] = 1.0
    b["gravity_enabled"] = 1
    b["allowed_to_sleep"] = 1
    return b


def collider_descs(n):
    c = np.zeros(n, COLLIDER_DESC_DTYPE)
    c["orientation"][:, 3] = 1.0
    c["friction"] = np.float32(0.3)
    c["bounciness"] = np.float32(0.5)
    c["mass_density"] = 1.0
    c["category"] = 1
    c["mask"] = 0xFFFF
    return c
