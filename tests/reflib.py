"""Loader for the oracles (test infrastructure).

- oracle/_ref/librp3d_ref_{f32,f64}.so: the reference engine itself, built
  from its sources by oracle/Makefile, driven through oracle/ref_harness.cpp.
- oracle/librp3d_oracle.so: the C restatement (oracle/rp3d_oracle.c).
Both take the rp3dg.h struct-of-arrays batches."""
import ctypes as C
import os

import numpy as np

from reactphysics3d_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_LIB = {"f32": os.path.join(ORACLE_DIR, "_ref", "librp3d_ref_f32.so"),
           "f64": os.path.join(ORACLE_DIR, "_ref", "librp3d_ref_f64.so")}
PORT_LIB = os.path.join(ORACLE_DIR, "librp3d_oracle.so")


def have_ref(prec="f32"):
    return os.path.exists(REF_LIB[prec])


class RefEngine:
    """The reference's own narrow-phase algorithms (FP32 or FP64 build)."""

    def __init__(self, prec="f32"):
        self.lib = C.CDLL(REF_LIB[prec])
        L = self.lib
        L.ref_narrowphase.argtypes = [C.c_int, C.c_void_p, C.c_uint32, C.POINTER(A.PairBatch),
                                      C.POINTER(A.ContactBatch), C.c_int, C.c_int, C.c_int,
                                      C.POINTER(C.c_double)]
        L.ref_create_convex_mesh.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                             C.POINTER(C.c_int32)]
        L.ref_create_convex_mesh_shape.argtypes = [C.c_int32, C.c_float, C.c_float, C.c_float,
                                                   C.POINTER(C.c_int32)]
        L.ref_get_convex_mesh_tables.argtypes = [C.c_int32] + [C.c_void_p] * 8 + [C.c_uint32, C.c_uint32]
        L.ref_quickhull.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                    C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p]

    def create_convex_mesh(self, vertices, faces):
        v = np.ascontiguousarray(vertices, dtype=np.float32)
        idx = np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint32) for f in faces]), dtype=np.uint32)
        sizes = np.array([len(f) for f in faces], dtype=np.uint32)
        out = C.c_int32()
        rc = self.lib.ref_create_convex_mesh(v.ctypes.data, len(v), idx.ctypes.data, sizes.ctypes.data,
                                             len(faces), C.byref(out))
        assert rc == 0, rc
        return out.value

    def create_convex_mesh_shape(self, mesh, scale=(1.0, 1.0, 1.0)):
        out = C.c_int32()
        rc = self.lib.ref_create_convex_mesh_shape(mesh, *map(float, scale), C.byref(out))
        assert rc == 0, rc
        return out.value

    def mesh_tables(self, instance, cap=4096):
        nv, nf, nh = C.c_uint32(), C.c_uint32(), C.c_uint32()
        he = np.zeros(4 * cap, np.uint32)
        fn = np.zeros(3 * cap, np.float32)
        fe = np.zeros(cap, np.uint32)
        cen = np.zeros(3, np.float32)
        verts = np.zeros(3 * cap, np.float32)
        rc = self.lib.ref_get_convex_mesh_tables(instance, C.addressof(nv), C.addressof(nf), C.addressof(nh),
                                                 he.ctypes.data, fn.ctypes.data, fe.ctypes.data,
                                                 cen.ctypes.data, verts.ctypes.data, cap, cap)
        assert rc == 0, rc
        return dict(half_edges=he[:4 * nh.value].reshape(-1, 4), face_normals=fn[:3 * nf.value].reshape(-1, 3),
                    face_edge=fe[:nf.value], centroid=cen, vertices=verts[:3 * nv.value].reshape(-1, 3))

    def quickhull(self, points):
        p = np.ascontiguousarray(points, dtype=np.float32)
        cap = 4096
        ov = np.zeros(3 * cap, np.float32)
        oi = np.zeros(4 * cap, np.uint32)
        osz = np.zeros(cap, np.uint32)
        nv, nf = C.c_uint32(), C.c_uint32()
        rc = self.lib.ref_quickhull(p.ctypes.data, len(p), ov.ctypes.data, cap, C.addressof(nv), oi.ctypes.data,
                                    4 * cap, osz.ctypes.data, cap, C.addressof(nf))
        assert rc == 0, rc
        verts = ov[:3 * nv.value].reshape(-1, 3).copy()
        faces, k = [], 0
        for s in osz[:nf.value]:
            faces.append([int(x) for x in oi[k:k + s]])
            k += int(s)
        return verts, faces

    def narrowphase(self, algo, shapes, pairs, out=None, clip=True, nthreads=1, repeats=1):
        """Run the reference algorithm; returns (HostContacts, seconds)."""
        if out is None:
            out = A.HostContacts(pairs.n)
        sh = np.ascontiguousarray(shapes)
        pb, cb = pairs.struct(), out.struct()
        sec = C.c_double()
        rc = self.lib.ref_narrowphase(algo, sh.ctypes.data, len(sh), C.byref(pb), C.byref(cb), int(clip),
                                      nthreads, repeats, C.byref(sec))
        assert rc == 0, rc
        return out, sec.value


class PortEngine:
    """The C restatement (oracle/rp3d_oracle.c) with the RefEngine interface."""

    def __init__(self):
        self.lib = C.CDLL(PORT_LIB)
        L = self.lib
        L.rp3do_narrowphase.argtypes = [C.c_int, C.c_void_p, C.c_uint32, C.POINTER(A.PairBatch),
                                        C.POINTER(A.ContactBatch), C.c_int]
        L.rp3do_create_convex_mesh.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                               C.POINTER(C.c_int32)]
        L.rp3do_create_convex_mesh_shape.argtypes = [C.c_int32, C.c_float, C.c_float, C.c_float,
                                                     C.POINTER(C.c_int32)]
        L.rp3do_get_convex_mesh_tables.argtypes = [C.c_int32] + [C.c_void_p] * 7 + [C.c_uint32, C.c_uint32]
        L.rp3do_reset()

    def create_convex_mesh(self, vertices, faces):
        v = np.ascontiguousarray(vertices, dtype=np.float32)
        idx = np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint32) for f in faces]), dtype=np.uint32)
        sizes = np.array([len(f) for f in faces], dtype=np.uint32)
        out = C.c_int32()
        rc = self.lib.rp3do_create_convex_mesh(v.ctypes.data, len(v), idx.ctypes.data, sizes.ctypes.data,
                                               len(faces), C.byref(out))
        assert rc == 0, rc
        return out.value

    def create_convex_mesh_shape(self, mesh, scale=(1.0, 1.0, 1.0)):
        out = C.c_int32()
        rc = self.lib.rp3do_create_convex_mesh_shape(mesh, *map(float, scale), C.byref(out))
        assert rc == 0, rc
        return out.value

    def mesh_tables(self, instance, cap=4096):
        nv, nf, nh = C.c_uint32(), C.c_uint32(), C.c_uint32()
        he = np.zeros(4 * cap, np.uint32)
        fn = np.zeros(3 * cap, np.float32)
        fe = np.zeros(cap, np.uint32)
        cen = np.zeros(3, np.float32)
        rc = self.lib.rp3do_get_convex_mesh_tables(instance, C.addressof(nv), C.addressof(nf), C.addressof(nh),
                                                   he.ctypes.data, fn.ctypes.data, fe.ctypes.data, cen.ctypes.data,
                                                   cap, cap)
        assert rc == 0, rc
        return dict(half_edges=he[:4 * nh.value].reshape(-1, 4), face_normals=fn[:3 * nf.value].reshape(-1, 3),
                    face_edge=fe[:nf.value], centroid=cen)

    def narrowphase(self, algo, shapes, pairs, out=None, clip=True):
        if out is None:
            out = A.HostContacts(pairs.n)
        sh = np.ascontiguousarray(shapes)
        pb, cb = pairs.struct(), out.struct()
        rc = self.lib.rp3do_narrowphase(algo, sh.ctypes.data, len(sh), C.byref(pb), C.byref(cb), int(clip))
        assert rc == 0, rc
        return out, 0.0


def compare_contacts(a, b, pairs_n):
    """Bit-level comparison of two HostContacts; returns a dict of mismatch counts."""
    res = {"is_colliding": int(np.sum(a.is_colliding != b.is_colliding)),
           "nb_contacts": int(np.sum(a.nb_contacts != b.nb_contacts))}
    same_nb = a.nb_contacts == b.nb_contacts
    mask = a.valid_mask() & same_nb[None, :]
    for f in ("normal_depth", "local1", "local2"):
        x = getattr(a, f).view(np.uint32)[mask]
        y = getattr(b, f).view(np.uint32)[mask]
        res[f] = int(np.sum(np.any(x != y, axis=-1)))
    return res


def perturb_pairs(pairs, rng, dpos=0.02, drot=0.02):
    """Small pose changes between two passes (exercises the temporal-coherence
    branches).  Quaternions are re-normalised in float64 then stored as float32."""
    q = A.HostPairs(pairs.shape1, pairs.shape2, pairs.pos1.copy(), pairs.rot1.copy(), pairs.pos2.copy(),
                    pairs.rot2.copy(), pairs.report, None if pairs.cache is None else pairs.cache.copy())
    n = pairs.n
    q.pos2[:, :3] += rng.uniform(-dpos, dpos, (n, 3)).astype(np.float32)
    r = q.rot2.astype(np.float64) + rng.uniform(-drot, drot, (n, 4))
    q.rot2[:] = (r / np.linalg.norm(r, axis=1, keepdims=True)).astype(np.float32)
    return q


def next_frame_cache(cache, out):
    """What the reference's collision detection does to a pair's cache between
    frames: the info becomes valid and remembers whether the pair collided
    (CollisionDetectionSystem::processPotentialContacts and
    OverlappingPairs::addLastFrameInfoIfNecessary)."""
    c = cache.copy()
    c["flags"] |= A.LF_IS_VALID
    c["flags"] &= ~np.uint8(A.LF_WAS_COLLIDING)
    c["flags"] |= np.where(out.is_colliding != 0, A.LF_WAS_COLLIDING, 0).astype(np.uint8)
    return c


def reduce_contacts(lib, fn, pairs, contacts):
    """Run a manifold-reduction entry point (ref_reduce_contacts or
    rp3do_reduce_contacts) in place; returns the kept-slot table (n x 4)."""
    getattr(lib, fn).argtypes = [C.POINTER(A.PairBatch), C.POINTER(A.ContactBatch), C.c_void_p]
    kept = np.zeros((pairs.n, 4), np.uint8)
    pb, cb = pairs.struct(), contacts.struct()
    rc = getattr(lib, fn)(C.byref(pb), C.byref(cb), kept.ctypes.data)
    assert rc == 0, rc
    return kept


def copy_contacts(c):
    d = A.HostContacts(c.n, c.max_contacts)
    for f in ("is_colliding", "nb_contacts", "normal_depth", "local1", "local2"):
        getattr(d, f)[...] = getattr(c, f)
    return d


# dtype of each captured dynamics field of oracle/ref_world.cpp, by suffix
_WORLD_DTYPES = {"body_gravity": np.uint8, "collider_body": np.int32, "manifold_ids": np.int32,
                 "manifold_point_start": np.uint32, "manifold_nb_points": np.uint8, "manifold_source": np.uint32,
                 "point_is_resting": np.uint8, "island_manifold_start": np.uint32,
                 "island_manifold_count": np.uint32, "body_nb_enabled": np.uint32,
                 "collider_nb_enabled": np.uint32, "bp_pairs": np.int32, "bp_bits": np.int32, "bp_id": np.int32,
                 "bp_moved": np.uint8, "dyn_seconds": np.float64}
_WORLD_SHAPES = {"manifold_ids": (-1, 4), "bp_pairs": (-1, 2), "bp_bits": (-1, 2), "point_penetration_impulse": (-1,), "body_inv_inertia_world": (-1, 3, 4),
                 "body_split_velocity": (-1, 2, 4)}


class RefWorld:
    """A reference world (oracle/ref_world.cpp) stepped by the reference; one
    step's dynamics stage can be captured as numpy arrays."""

    def __init__(self, kind=1, seed=1, nx=4, ny=3, nz=4, spacing=1.6, variety=True, prec="f32"):
        self.lib = C.CDLL(REF_LIB[prec])
        L = self.lib
        L.ref_world_create.argtypes = [C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int]
        L.ref_world_apply_forces.argtypes = [C.c_int, C.c_uint64]
        L.ref_world_step.argtypes = [C.c_int, C.c_float, C.c_int]
        L.ref_world_capture.argtypes = [C.c_int, C.c_float]
        L.ref_world_field_size.argtypes = [C.c_int, C.c_char_p]
        L.ref_world_field_size.restype = C.c_long
        L.ref_world_field.argtypes = [C.c_int, C.c_char_p, C.c_void_p]
        L.ref_world_field_names.argtypes = [C.c_int, C.c_char_p, C.c_int]
        self.id = L.ref_world_create(kind, seed, nx, ny, nz, spacing, int(variety))

    def step(self, dt=1.0 / 60.0, n=1):
        self.lib.ref_world_step(self.id, dt, n)

    def apply_forces(self, seed):
        self.lib.ref_world_apply_forces(self.id, seed)

    def capture(self, dt=1.0 / 60.0):
        """One step, phase by phase; returns {name: array} of the dynamics
        stage's inputs (in_*), outputs (out_*) and params."""
        assert self.lib.ref_world_capture(self.id, dt) == 0
        buf = C.create_string_buffer(1 << 16)
        assert self.lib.ref_world_field_names(self.id, buf, len(buf)) == 0
        out = {}
        for name in buf.value.decode().split():
            size = self.lib.ref_world_field_size(self.id, name.encode())
            suffix = name.split("_", 1)[1] if name.startswith(("in_", "out_")) else name
            dt_ = _WORLD_DTYPES.get(suffix, np.float32)
            a = np.zeros(size // np.dtype(dt_).itemsize, dt_)
            assert self.lib.ref_world_field(self.id, name.encode(), a.ctypes.data) == 0
            if suffix in _WORLD_SHAPES:
                a = a.reshape(_WORLD_SHAPES[suffix])
            elif dt_ == np.float32 and suffix != "params":
                a = a.reshape(-1, 4)
            out[name] = a
        return out


def concave_register(L, vertices, triangles, normals, scale):
    """Register a triangle mesh + scale with the reference harness; returns its id."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
    n = None if normals is None else np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
    return L.ref_concave_register(v.ctypes.data, len(v), t.ctypes.data, len(t), None if n is None else n.ctypes.data,
                                  *map(float, scale))


def ref_triangle_mesh(vertices, triangles, normals=None, prec="f32"):
    """TriangleMesh of the reference build over these arrays: (vertices,
    vertex normals, triangles), or None where the reference rejects it."""
    L = C.CDLL(REF_LIB[prec])
    P = C.c_void_p
    L.ref_concave_register.argtypes = [P, C.c_uint32, P, C.c_uint32, P, C.c_float, C.c_float, C.c_float]
    L.ref_concave_mesh_data.argtypes = [C.c_int, P, P, P, C.c_uint32, C.c_uint32, P, P]
    cid = concave_register(L, vertices, triangles, normals, (1.0, 1.0, 1.0))
    nv, nt = C.c_uint32(), C.c_uint32()
    if L.ref_concave_mesh_data(cid, None, None, None, 0, 0, C.byref(nv), C.byref(nt)) != 0:
        return None
    v = np.zeros((nv.value, 3), np.float32)
    n = np.zeros((nv.value, 3), np.float32)
    t = np.zeros((nt.value, 3), np.uint32)
    L.ref_concave_mesh_data(cid, v.ctypes.data, n.ctypes.data, t.ctypes.data, len(v), len(t), C.byref(nv), C.byref(nt))
    return v, n, t


class RefScene:
    """A reference world built from a scenes.WorldScene (oracle/ref_world.cpp
    ref_scene_create, the call sequence of rp3dg_world_create) and stepped by
    PhysicsWorld::update."""

    def __init__(self, scene, prec="f32"):
        self.lib = C.CDLL(REF_LIB[prec])
        L = self.lib
        P = C.c_void_p
        L.ref_scene_create.argtypes = [P, P, C.c_uint32, P, C.c_uint32, P, C.c_uint32]
        L.ref_scene_bodies.argtypes = [C.c_int, P, P, P, P, P]
        L.ref_scene_pairs.argtypes = [C.c_int, P, C.c_long]
        L.ref_scene_pairs.restype = C.c_long
        L.ref_scene_contacts.argtypes = [C.c_int, P, P, P, C.c_long, P, P, P, C.c_long, C.POINTER(C.c_long)]
        L.ref_scene_contacts.restype = C.c_long
        L.ref_world_step.argtypes = [C.c_int, C.c_float, C.c_int]
        L.ref_scene_add_joints.argtypes = [C.c_int, P, C.c_uint32]
        L.ref_scene_set_motor_speed.argtypes = [C.c_int, C.c_uint32, C.c_float]
        L.ref_scene_raycast.argtypes = [C.c_int, P, C.c_uint32, C.c_int, C.c_uint32, P, P]
        L.ref_scene_events.argtypes = [C.c_int, P, C.c_uint32, P, P, P, C.c_uint32, P, P]
        L.ref_scene_trigger_events.argtypes = [C.c_int, P, C.c_uint32, P]
        L.ref_scene_set_debug.argtypes = [C.c_int, C.c_uint32]
        L.ref_scene_set_body_debug.argtypes = [C.c_int, C.c_int, C.c_int]
        L.ref_scene_debug_primitives.argtypes = [C.c_int, P, C.c_uint32, P, C.c_uint32, P, P]
        L.ref_convex_register.argtypes = [P, C.c_uint32, P, P, C.c_uint32, C.c_float, C.c_float, C.c_float]
        L.ref_heightfield_register.argtypes = [C.c_uint32, C.c_uint32, P, C.c_float, C.c_float, C.c_float]
        L.ref_concave_register.argtypes = [P, C.c_uint32, P, C.c_uint32, P, C.c_float, C.c_float, C.c_float]
        # height fields of the scene registered with the harness; the shape
        # table's mesh field then names the harness's ids
        shapes = np.array(scene.shapes, copy=True)
        hf_ids = []
        for heights, scale in getattr(scene, "heightfields", None) or []:
            h = np.ascontiguousarray(heights, dtype=np.float32)
            hf_ids.append(L.ref_heightfield_register(h.shape[1], h.shape[0], h.ctypes.data, *map(float, scale)))
        for i in np.nonzero(shapes["kind"] == A.SHAPE_HEIGHTFIELD)[0]:
            shapes["mesh"][i] = hf_ids[int(shapes["mesh"][i])]
        cm_ids = []
        for v, faces, scale in getattr(scene, "convex_meshes", None) or []:
            v = np.ascontiguousarray(v, dtype=np.float32)
            idx = np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint32) for f in faces]), dtype=np.uint32)
            sizes = np.array([len(f) for f in faces], dtype=np.uint32)
            cm_ids.append(L.ref_convex_register(v.ctypes.data, len(v), idx.ctypes.data, sizes.ctypes.data,
                                                len(faces), *map(float, scale)))
        for i in np.nonzero(shapes["kind"] == A.SHAPE_CONVEX_MESH)[0]:
            shapes["mesh"][i] = cm_ids[int(shapes["mesh"][i])]
        cc_ids = [concave_register(L, *m) for m in getattr(scene, "concave_meshes", None) or []]
        for i in np.nonzero(shapes["kind"] == A.SHAPE_CONCAVE_MESH)[0]:
            shapes["mesh"][i] = cc_ids[int(shapes["mesh"][i])]
        self._keep = (np.ascontiguousarray(scene.settings).copy(), np.ascontiguousarray(shapes),
                      np.ascontiguousarray(scene.bodies), np.ascontiguousarray(scene.colliders))
        st, sh, bd, cd = self._keep
        self.id = L.ref_scene_create(st.ctypes.data, sh.ctypes.data, len(sh), bd.ctypes.data, len(bd),
                                     cd.ctypes.data, len(cd))
        assert self.id >= 0
        self.nb = len(bd)
        joints = getattr(scene, "joints", None)
        if joints is not None and len(joints):
            self._joints = np.ascontiguousarray(joints)
            assert L.ref_scene_add_joints(self.id, self._joints.ctypes.data, len(self._joints)) == 0

    def update(self, dt=1.0 / 60.0, n=1):
        self.lib.ref_world_step(self.id, dt, n)

    def contact_events(self):
        ne, npt = C.c_uint32(), C.c_uint32()
        self.lib.ref_scene_events(self.id, None, 0, None, None, None, 0, C.byref(ne), C.byref(npt))
        ev = np.zeros(ne.value, A.CONTACT_EVENT_DTYPE)
        nd, l1, l2 = (np.zeros((npt.value, 4), np.float32) for _ in range(3))
        self.lib.ref_scene_events(self.id, ev.ctypes.data, len(ev), nd.ctypes.data, l1.ctypes.data, l2.ctypes.data,
                                  len(nd), C.byref(ne), C.byref(npt))
        return ev, nd, l1, l2

    def trigger_events(self):
        n = C.c_uint32()
        self.lib.ref_scene_trigger_events(self.id, None, 0, C.byref(n))
        ev = np.zeros(n.value, A.CONTACT_EVENT_DTYPE)
        self.lib.ref_scene_trigger_events(self.id, ev.ctypes.data if len(ev) else None, len(ev), C.byref(n))
        return ev

    def set_debug_rendering(self, items=A.DEBUG_ALL):
        self.lib.ref_scene_set_debug(self.id, int(items))

    def set_body_debug(self, body=-1, enabled=True):
        self.lib.ref_scene_set_body_debug(self.id, int(body), int(bool(enabled)))

    def debug_primitives(self):
        nl, nt = C.c_uint32(), C.c_uint32()
        self.lib.ref_scene_debug_primitives(self.id, None, 0, None, 0, C.byref(nl), C.byref(nt))
        lines = np.zeros(nl.value, A.DEBUG_LINE_DTYPE)
        tris = np.zeros(nt.value, A.DEBUG_TRIANGLE_DTYPE)
        self.lib.ref_scene_debug_primitives(self.id, lines.ctypes.data if len(lines) else None, len(lines),
                                            tris.ctypes.data if len(tris) else None, len(tris), C.byref(nl), C.byref(nt))
        return lines, tris

    def raycast(self, rays, mode=A.RAYCAST_CLOSEST, max_hits=1):
        r = np.ascontiguousarray(rays, dtype=A.RAY_DTYPE)
        n = len(r)
        hits = np.zeros((n, max_hits), A.RAYCAST_HIT_DTYPE)
        counts = np.zeros(n, np.uint32)
        assert self.lib.ref_scene_raycast(self.id, r.ctypes.data, n, int(mode), int(max_hits), hits.ctypes.data,
                                          counts.ctypes.data) == 0
        return hits, counts

    def set_motor_speed(self, joint, speed):
        assert self.lib.ref_scene_set_motor_speed(self.id, int(joint), float(speed)) == 0

    def bodies(self):
        n = self.nb
        p, q = np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32)
        lv, av = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
        sl = np.zeros(n, np.uint8)
        self.lib.ref_scene_bodies(self.id, p.ctypes.data, q.ctypes.data, lv.ctypes.data, av.ctypes.data, sl.ctypes.data)
        return p, q, lv, av, sl

    def pairs(self):
        n = self.lib.ref_scene_pairs(self.id, None, 0)
        out = np.zeros(n, np.uint64)
        self.lib.ref_scene_pairs(self.id, out.ctypes.data, n)
        return out

    def contacts(self):
        npt = C.c_long()
        nm = self.lib.ref_scene_contacts(self.id, None, None, None, 0, None, None, None, 0, C.byref(npt))
        b1, b2 = np.zeros(nm, np.int32), np.zeros(nm, np.int32)
        k = np.zeros(nm, np.uint8)
        nd, l1, l2 = (np.zeros((npt.value, 4), np.float32) for _ in range(3))
        self.lib.ref_scene_contacts(self.id, b1.ctypes.data, b2.ctypes.data, k.ctypes.data, nm, nd.ctypes.data,
                                    l1.ctypes.data, l2.ctypes.data, npt.value, C.byref(npt))
        return b1, b2, k, nd, l1, l2
