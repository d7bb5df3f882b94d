"""Python binding of the C ABI (include/rp3dg.h) of librp3dg.so.

`Context` owns one rp3dg_ctx (one CUDA device, one stream).  Batches can be
given as numpy arrays in host memory (`narrowphase_host`, the call a CPU-side
engine would make in place of XxxAlgorithm::testCollision) or as torch CUDA
tensors already resident in device memory (`narrowphase_device`).

There is no CPU fallback: if the library is missing or no GPU is present the
calls raise.
"""
import ctypes as C
import os
import re

import numpy as np

from . import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "librp3dg.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "rp3dg.h")

RP3DG_OK, RP3DG_EINVAL, RP3DG_ECUDA, RP3DG_ENOMEM, RP3DG_ECAPACITY, RP3DG_ENODEV = 0, -1, -2, -3, -4, -5
NP_EVENTS = 40  # RP3DG_NP_EVENTS

_lib = None


SOLVER_EXACT, SOLVER_GRAPH_COLORED = 0, 1


class SolverStats(C.Structure):
    """rp3dg_solver_stats (include/rp3dg.h)."""
    _fields_ = [("residual_rms", C.c_double), ("residual_max", C.c_double), ("kinetic_energy", C.c_double),
                ("potential_energy", C.c_double), ("contact_points", C.c_uint32), ("colors", C.c_uint32),
                ("coloring_rounds", C.c_uint32), ("reserved", C.c_uint32)]


class Rp3dgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rp3dg error {code}: {msg}")
        self.code = code


def declared_symbols(header=HEADER):
    """Function names declared in include/rp3dg.h."""
    text = open(header).read()
    return sorted(set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(rp3dg_\w+)\s*\(", text, re.M)))


def load_library(path=LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m reactphysics3d_b200.build` "
                                "(there is no CPU fallback)")
    L = C.CDLL(path)
    P = C.c_void_p
    L.rp3dg_create.argtypes = [C.c_int, C.POINTER(P)]
    L.rp3dg_destroy.argtypes = [P]
    L.rp3dg_destroy.restype = None
    L.rp3dg_last_error.argtypes = [P]
    L.rp3dg_last_error.restype = C.c_char_p
    L.rp3dg_stream.argtypes = [P]
    L.rp3dg_stream.restype = P
    L.rp3dg_synchronize.argtypes = [P]
    L.rp3dg_kernel_launches.argtypes = [P]
    L.rp3dg_kernel_launches.restype = C.c_uint64
    L.rp3dg_create_convex_mesh.argtypes = [P, P, C.c_uint32, P, P, C.c_uint32, C.POINTER(C.c_int32)]
    L.rp3dg_create_convex_mesh_shape.argtypes = [P, C.c_int32, C.c_float, C.c_float, C.c_float,
                                                 C.POINTER(C.c_int32)]
    L.rp3dg_get_convex_mesh_tables.argtypes = [P, C.c_int32] + [P] * 7 + [C.c_uint32, C.c_uint32]
    L.rp3dg_set_shapes.argtypes = [P, P, C.c_uint32]
    L.rp3dg_create_heightfield.argtypes = [P, C.c_uint32, C.c_uint32, P, C.c_float, C.c_float, C.c_float,
                                           C.POINTER(C.c_int32)]
    L.rp3dg_create_triangle_mesh.argtypes = [P, P, C.c_uint32, P, C.c_uint32, P, C.POINTER(C.c_int32)]
    L.rp3dg_create_concave_mesh_shape.argtypes = [P, C.c_int32, C.c_float, C.c_float, C.c_float,
                                                  C.POINTER(C.c_int32)]
    L.rp3dg_get_triangle_mesh.argtypes = [P, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), P, P, P,
                                          C.c_uint32, C.c_uint32]
    L.rp3dg_device_errors.argtypes = [P, C.POINTER(C.c_uint32), C.c_int]
    L.rp3dg_narrowphase_device.argtypes = [P, C.c_int, C.POINTER(A.PairBatch), C.POINTER(A.ContactBatch), C.c_int]
    L.rp3dg_narrowphase_host.argtypes = [P, C.c_int, C.POINTER(A.PairBatch), C.POINTER(A.ContactBatch), C.c_int]
    L.rp3dg_narrowphase_input_host.argtypes = [P, C.c_uint32, P, P, P, C.c_int]
    L.rp3dg_narrowphase_count_events.argtypes = [P, C.c_int, C.POINTER(A.PairBatch), C.POINTER(A.ContactBatch),
                                                 C.c_int, C.POINTER(C.c_ulonglong)]
    L.rp3dg_measure_fp32_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.rp3dg_reduce_contacts_device.argtypes = [P, C.POINTER(A.PairBatch), C.POINTER(A.ContactBatch), P]
    L.rp3dg_narrowphase_manifolds_host.argtypes = [P, C.c_int, C.POINTER(A.PairBatch), C.POINTER(A.ContactBatch),
                                                   C.c_int, P]
    from . import broadphase as BP
    BP.bind(L)
    from . import dynamics as DY
    for fn in ("rp3dg_dynamics_step_host", "rp3dg_dynamics_step_device"):
        getattr(L, fn).argtypes = [P, C.POINTER(DY.Params), C.POINTER(DY.Bodies), C.POINTER(DY.Colliders),
                                   C.POINTER(DY.Manifolds), C.POINTER(DY.Points), C.POINTER(DY.Islands)]
    L.rp3dg_axis_mlp_init.argtypes = [P, C.c_uint64]
    L.rp3dg_axis_mlp_get_params.argtypes = [P, P]
    L.rp3dg_axis_mlp_set_params.argtypes = [P, P]
    L.rp3dg_axis_features.argtypes = [P, C.POINTER(A.PairBatch), P]
    L.rp3dg_axis_labels.argtypes = [P, C.POINTER(A.PairBatch), P, P]
    L.rp3dg_axis_mlp_grads.argtypes = [P, P, P, C.c_uint32, P, P]
    L.rp3dg_axis_mlp_train_step.argtypes = [P, P, P, C.c_uint32, C.c_float, P]
    L.rp3dg_axis_mlp_predict.argtypes = [P, P, C.c_uint32, P]
    L.rp3dg_set_learned_axis.argtypes = [P, C.c_int]
    L.rp3dg_learned_axis_stats.argtypes = [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_int]
    L.rp3dg_world_create.argtypes = [P, P, P, C.c_uint32, P, C.c_uint32, C.POINTER(P)]
    L.rp3dg_world_destroy.argtypes = [P]
    L.rp3dg_world_destroy.restype = None
    L.rp3dg_world_update.argtypes = [P, C.c_float]
    L.rp3dg_world_get_bodies.argtypes = [P, P, P, P, P, P]
    L.rp3dg_world_get_pairs.argtypes = [P, P, C.c_uint32, C.POINTER(C.c_uint32)]
    L.rp3dg_world_get_contacts.argtypes = [P, P, P, P, C.c_uint32, P, P, P, C.c_uint32,
                                           C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.rp3dg_world_get_stats.argtypes = [P, P]
    L.rp3dg_world_set_profiling.argtypes = [P, C.c_int]
    L.rp3dg_world_set_threads.argtypes = [P, C.c_int]
    L.rp3dg_world_set_device_trees.argtypes = [P, C.c_int]
    L.rp3dg_world_get_device_trees.argtypes = [P, P]
    L.rp3dg_world_autotune.argtypes = [P, C.c_int]
    L.rp3dg_world_get_tuning.argtypes = [P, P]
    L.rp3dg_world_add_joints.argtypes = [P, P, C.c_uint32]
    L.rp3dg_world_group_add_joints.argtypes = [P, C.c_uint32, P, C.c_uint32]
    L.rp3dg_world_set_motor_speed.argtypes = [P, C.c_uint32, C.c_uint32, C.c_float]
    L.rp3dg_world_get_contact_events.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P, P, C.c_uint32,
                                                 C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.rp3dg_world_get_trigger_events.argtypes = [P, C.c_uint32, P, C.c_uint32, C.POINTER(C.c_uint32)]
    L.rp3dg_world_set_debug_rendering.argtypes = [P, C.c_uint32]
    L.rp3dg_world_set_body_debug.argtypes = [P, C.c_uint32, C.c_int32, C.c_int]
    L.rp3dg_world_get_debug_primitives.argtypes = [P, C.c_uint32, P, C.c_uint32, P, C.c_uint32,
                                                   C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_int]
    L.rp3dg_world_raycast.argtypes = [P, C.c_uint32, P, C.c_uint32, C.c_int32, C.c_uint32, P, P]
    L.rp3dg_world_raycast_device.argtypes = [P, C.c_uint32, P, C.c_uint32, C.c_int32, C.c_uint32, P, P,
                                             C.POINTER(C.c_float)]
    L.rp3dg_world_group_create.argtypes = [P, P, C.c_uint32, P, P, P, P, C.c_int, C.POINTER(P)]
    L.rp3dg_world_group_get_bodies.argtypes = [P, C.c_uint32, P, P, P, P, P]
    L.rp3dg_world_group_get_pairs.argtypes = [P, C.c_uint32, P, C.c_uint32, C.POINTER(C.c_uint32)]
    L.rp3dg_world_group_get_contacts.argtypes = [P, C.c_uint32, P, P, P, C.c_uint32, P, P, P, C.c_uint32,
                                                 C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.rp3dg_world_get_phase_times.argtypes = [P, P, C.c_uint32]
    L.rp3dg_world_set_solver.argtypes = [P, C.c_int, C.c_int]
    L.rp3dg_world_get_solver_stats.argtypes = [P, C.POINTER(SolverStats)]
    _lib = L
    return L


class DevicePairs:
    """A pair batch resident in device memory (torch CUDA tensors)."""

    def __init__(self, host_pairs, device="cuda"):
        import torch
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        h = host_pairs
        self.n = h.n
        self.shape1, self.shape2 = t(h.shape1), t(h.shape2)
        self.pos1, self.rot1, self.pos2, self.rot2 = t(h.pos1), t(h.rot1), t(h.pos2), t(h.rot2)
        self.report = None if h.report is None else t(h.report)
        self.cache = None if h.cache is None else t(h.cache.view(np.uint8).reshape(-1, 16))

    def struct(self):
        p = lambda x: None if x is None else x.data_ptr()
        return A.PairBatch(self.n, p(self.shape1), p(self.shape2), p(self.pos1), p(self.rot1), p(self.pos2),
                           p(self.rot2), p(self.report), p(self.cache))

    def host_cache(self):
        return None if self.cache is None else self.cache.cpu().numpy().reshape(-1).view(A.CACHE_DTYPE)


class DeviceContacts:
    """Narrow-phase results in device memory (torch CUDA tensors)."""

    def __init__(self, n, max_contacts=A.MAX_CONTACTS, device="cuda"):
        import torch
        self.n, self.max_contacts = n, max_contacts
        self.is_colliding = torch.zeros(n, dtype=torch.uint8, device=device)
        self.nb_contacts = torch.zeros(n, dtype=torch.uint8, device=device)
        self.normal_depth = torch.zeros((max_contacts, n, 4), dtype=torch.float32, device=device)
        self.local1 = torch.zeros((max_contacts, n, 4), dtype=torch.float32, device=device)
        self.local2 = torch.zeros((max_contacts, n, 4), dtype=torch.float32, device=device)

    def struct(self):
        return A.ContactBatch(self.is_colliding.data_ptr(), self.nb_contacts.data_ptr(),
                              self.normal_depth.data_ptr(), self.local1.data_ptr(), self.local2.data_ptr(),
                              self.max_contacts)

    def to_host(self):
        h = A.HostContacts(self.n, self.max_contacts)
        h.is_colliding[:] = self.is_colliding.cpu().numpy()
        h.nb_contacts[:] = self.nb_contacts.cpu().numpy()
        h.normal_depth[:] = self.normal_depth.cpu().numpy()
        h.local1[:] = self.local1.cpu().numpy()
        h.local2[:] = self.local2.cpu().numpy()
        return h


class Context:
    """One rp3dg_ctx: device, stream, shape and mesh tables."""

    def __init__(self, device=0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.rp3dg_create(int(device), C.byref(h))
        if rc != 0:
            raise Rp3dgError(rc, "rp3dg_create failed (no CUDA device?)")
        self.h = h
        self.device = device
        self._shapes = None

    def close(self):
        if self.h:
            self.lib.rp3dg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.h).decode())

    @property
    def stream_ptr(self):
        return self.lib.rp3dg_stream(self.h)

    def torch_stream(self):
        import torch
        if getattr(self, "_tstream", None) is None:
            self._tstream = torch.cuda.ExternalStream(self.stream_ptr, device=f"cuda:{self.device}")
        return self._tstream

    def order_in(self):
        """Make the context stream wait for work queued on torch's current
        stream (tensors just created or filled there)."""
        import torch
        cur = torch.cuda.current_stream(self.device)
        if cur.cuda_stream != self.stream_ptr:
            ev = torch.cuda.Event()
            ev.record(cur)
            self.torch_stream().wait_event(ev)

    def order_out(self):
        """Make torch's current stream wait for the context stream (results
        read or reused there)."""
        import torch
        cur = torch.cuda.current_stream(self.device)
        if cur.cuda_stream != self.stream_ptr:
            ev = torch.cuda.Event()
            ev.record(self.torch_stream())
            cur.wait_event(ev)

    def synchronize(self):
        self._check(self.lib.rp3dg_synchronize(self.h))

    def device_errors(self, clear=True):
        f = C.c_uint32()
        self._check(self.lib.rp3dg_device_errors(self.h, C.byref(f), int(clear)))
        return f.value

    def kernel_launches(self):
        return int(self.lib.rp3dg_kernel_launches(self.h))

    def create_convex_mesh(self, vertices, faces):
        v = np.ascontiguousarray(vertices, dtype=np.float32)
        idx = np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint32) for f in faces]), dtype=np.uint32)
        sizes = np.array([len(f) for f in faces], dtype=np.uint32)
        out = C.c_int32()
        self._check(self.lib.rp3dg_create_convex_mesh(self.h, v.ctypes.data, len(v), idx.ctypes.data,
                                                      sizes.ctypes.data, len(faces), C.byref(out)))
        return out.value

    def create_convex_mesh_shape(self, mesh, scale=(1.0, 1.0, 1.0)):
        out = C.c_int32()
        self._check(self.lib.rp3dg_create_convex_mesh_shape(self.h, mesh, *map(float, scale), C.byref(out)))
        return out.value

    def create_heightfield(self, heights, scale=(1.0, 1.0, 1.0)):
        """Height field from an (nb_rows, nb_columns) float32 grid (row y
        along local Z, column x along local X); returns the id for
        rp3dg_shape.mesh with kind SHAPE_HEIGHTFIELD."""
        h = np.ascontiguousarray(heights, dtype=np.float32)
        assert h.ndim == 2
        out = C.c_int32()
        self._check(self.lib.rp3dg_create_heightfield(self.h, h.shape[1], h.shape[0], h.ctypes.data,
                                                      *map(float, scale), C.byref(out)))
        return out.value

    def create_triangle_mesh(self, vertices, triangles, normals=None):
        """PhysicsCommon::createTriangleMesh over float vertices (n, 3),
        uint32 triangles (m, 3) and optional vertex normals (n, 3); returns
        the mesh id."""
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        n = None if normals is None else np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
        out = C.c_int32()
        self._check(self.lib.rp3dg_create_triangle_mesh(self.h, v.ctypes.data, len(v), t.ctypes.data, len(t),
                                                        None if n is None else n.ctypes.data, C.byref(out)))
        return out.value

    def create_concave_mesh_shape(self, mesh, scale=(1.0, 1.0, 1.0)):
        """PhysicsCommon::createConcaveMeshShape; returns the instance id for
        rp3dg_shape.mesh with kind SHAPE_CONCAVE_MESH."""
        out = C.c_int32()
        self._check(self.lib.rp3dg_create_concave_mesh_shape(self.h, mesh, *map(float, scale), C.byref(out)))
        return out.value

    def triangle_mesh(self, mesh):
        """The mesh as built: (vertices (n, 3), vertex normals (n, 3), triangles (m, 3))."""
        nv, nt = C.c_uint32(), C.c_uint32()
        self._check(self.lib.rp3dg_get_triangle_mesh(self.h, mesh, C.byref(nv), C.byref(nt), None, None, None, 0, 0))
        v = np.zeros((nv.value, 3), np.float32)
        n = np.zeros((nv.value, 3), np.float32)
        t = np.zeros((nt.value, 3), np.uint32)
        self._check(self.lib.rp3dg_get_triangle_mesh(self.h, mesh, C.byref(nv), C.byref(nt), v.ctypes.data,
                                                     n.ctypes.data, t.ctypes.data, len(v), len(t)))
        return v, n, t

    def scene_shapes(self, scene):
        """The scene's shape table with its height fields created in this
        context (scene.heightfields: list of (heights, scale); a height-field
        shape's mesh field indexes that list)."""
        shapes = np.array(scene.shapes, copy=True)
        hfs = getattr(scene, "heightfields", None) or []
        ids = [self.create_heightfield(h, s) for (h, s) in hfs]
        for i in np.nonzero(shapes["kind"] == A.SHAPE_HEIGHTFIELD)[0]:
            shapes["mesh"][i] = ids[int(shapes["mesh"][i])]
        # convex meshes (scene.convex_meshes: list of (vertices, faces, scale);
        # a convex-mesh shape's mesh field indexes that list)
        cms = getattr(scene, "convex_meshes", None) or []
        inst = [self.create_convex_mesh_shape(self.create_convex_mesh(v, f), s) for (v, f, s) in cms]
        for i in np.nonzero(shapes["kind"] == A.SHAPE_CONVEX_MESH)[0]:
            shapes["mesh"][i] = inst[int(shapes["mesh"][i])]
        # concave meshes (scene.concave_meshes: list of (vertices, triangles,
        # normals or None, scale); a concave-mesh shape's mesh field indexes
        # that list)
        ccs = getattr(scene, "concave_meshes", None) or []
        cinst = [self.create_concave_mesh_shape(self.create_triangle_mesh(v, t, n), s) for (v, t, n, s) in ccs]
        for i in np.nonzero(shapes["kind"] == A.SHAPE_CONCAVE_MESH)[0]:
            shapes["mesh"][i] = cinst[int(shapes["mesh"][i])]
        return shapes

    def mesh_tables(self, instance, cap=4096):
        nv, nf, nh = C.c_uint32(), C.c_uint32(), C.c_uint32()
        he = np.zeros(4 * cap, np.uint32)
        fn = np.zeros(3 * cap, np.float32)
        fe = np.zeros(cap, np.uint32)
        cen = np.zeros(3, np.float32)
        self._check(self.lib.rp3dg_get_convex_mesh_tables(self.h, instance, C.addressof(nv), C.addressof(nf),
                                                          C.addressof(nh), he.ctypes.data, fn.ctypes.data,
                                                          fe.ctypes.data, cen.ctypes.data, cap, cap))
        return dict(half_edges=he[:4 * nh.value].reshape(-1, 4), face_normals=fn[:3 * nf.value].reshape(-1, 3),
                    face_edge=fe[:nf.value], centroid=cen)

    def set_shapes(self, shapes):
        sh = np.ascontiguousarray(shapes, dtype=A.SHAPE_DTYPE)
        self._check(self.lib.rp3dg_set_shapes(self.h, sh.ctypes.data, len(sh)))
        self._shapes = sh

    def narrowphase_host(self, algo, pairs, out=None, clip=True):
        if out is None:
            out = A.HostContacts(pairs.n)
        pb, cb = pairs.struct(), out.struct()
        self._check(self.lib.rp3dg_narrowphase_host(self.h, int(algo), C.byref(pb), C.byref(cb), int(clip)))
        return out

    def narrowphase_input_host(self, batches, clip=True):
        """testNarrowPhaseCollision over a whole NarrowPhaseInput: `batches` is
        a list of (algorithm, HostPairs, HostContacts or None); the batches
        run overlapped (rp3dg_narrowphase_input_host); returns the outputs."""
        return self.narrowphase_input_call(batches, clip)()

    def narrowphase_input_call(self, batches, clip=True):
        """The same call prepared once for fixed host arrays (their contents
        may change between runs): returns a function that makes one
        rp3dg_narrowphase_input_host call and returns the outputs, without
        rebuilding the batch descriptors each time."""
        outs = [o if o is not None else A.HostContacts(p.n) for (_, p, o) in batches]
        n = len(batches)
        algos = (C.c_int32 * n)(*[int(a) for (a, _, _) in batches])
        pbs = (A.PairBatch * n)(*[p.struct() for (_, p, _) in batches])
        cbs = (A.ContactBatch * n)(*[o.struct() for o in outs])
        fn, h, args = self.lib.rp3dg_narrowphase_input_host, self.h, (C.addressof(algos), C.addressof(pbs),
                                                                       C.addressof(cbs), int(clip))
        keep = (algos, pbs, cbs, batches)

        def run():
            rc = fn(h, n, *args)
            if rc != 0:
                self._check(rc)
            return outs
        run.keep = keep
        return run

    def narrowphase_manifolds_host(self, algo, pairs, out=None, clip=True, want_kept=True):
        """Narrow phase + manifold reduction on host arrays; returns (out, kept)."""
        out = out if out is not None else A.HostContacts(pairs.n)
        kept = np.zeros((pairs.n, 4), np.uint8) if want_kept else None
        pb, cb = pairs.struct(), out.struct()
        self._check(self.lib.rp3dg_narrowphase_manifolds_host(self.h, algo, C.byref(pb), C.byref(cb), int(clip),
                                                              None if kept is None else kept.ctypes.data))
        return out, kept

    def broadphase_update(self, bp):
        """Fat-AABB update on device arrays (reactphysics3d_b200.broadphase.make)."""
        self.order_in()
        self._check(self.lib.rp3dg_broadphase_update_device(self.h, C.byref(bp)))
        self.order_out()

    def broadphase_pairs(self, bp, capacity, axis=-1, device=False):
        """Overlapping pairs: (count, pairs (capacity x 2 int32)).  Host arrays
        unless device is set (then pairs and the count are CUDA tensors)."""
        if device:
            import torch
            pairs = torch.empty((max(capacity, 1), 2), dtype=torch.int32, device="cuda")
            cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
            self.order_in()
            self._check(self.lib.rp3dg_broadphase_pairs_device(self.h, C.byref(bp), axis, pairs.data_ptr(), capacity,
                                                               cnt.data_ptr()))
            self.order_out()
            return cnt, pairs
        pairs = np.zeros((max(capacity, 1), 2), np.int32)
        cnt = C.c_uint32(0)
        self._check(self.lib.rp3dg_broadphase_pairs_host(self.h, C.byref(bp), axis, pairs.ctypes.data, capacity,
                                                         C.addressof(cnt)))
        return int(cnt.value), pairs

    def dynamics_step(self, params, world):
        """One dynamics stage (inertia, velocities, contact solver, positions,
        state) on a reactphysics3d_b200.dynamics.DynWorld, in place: host
        arrays through rp3dg_dynamics_step_host, CUDA tensors through
        rp3dg_dynamics_step_device (asynchronous)."""
        b, c, m, p, i = world.structs()
        if world.device is None:
            fn = self.lib.rp3dg_dynamics_step_host
        else:
            fn = self.lib.rp3dg_dynamics_step_device
            self.order_in()
        self._check(fn(self.h, C.byref(params), C.byref(b), C.byref(c), C.byref(m), C.byref(p), C.byref(i)))
        if world.device is not None:
            self.order_out()
        return world

    def reduce_contacts_device(self, pairs, contacts, kept=None):
        """Convex-pair manifold reduction in place on DeviceContacts; kept is an
        optional (n, 4) uint8 CUDA tensor receiving the kept slots."""
        pb, cb = pairs.struct(), contacts.struct()
        self.order_in()
        self._check(self.lib.rp3dg_reduce_contacts_device(self.h, C.byref(pb), C.byref(cb),
                                                          None if kept is None else kept.data_ptr()))
        self.order_out()
        return contacts

    def narrowphase_count_events(self, algo, pairs, out, clip=True):
        """Run a device batch through the event-counting build of the kernels;
        returns the RP3DG_NP_EVENTS path-event counts (numpy uint64)."""
        ev = (C.c_ulonglong * NP_EVENTS)()
        pb, cb = pairs.struct(), out.struct()
        self._check(self.lib.rp3dg_narrowphase_count_events(self.h, int(algo), C.byref(pb), C.byref(cb), int(clip), ev))
        return np.array(ev[:], dtype=np.uint64)

    def measure_fp32_peak(self, fused=False):
        """FP32 operations per second of this context's device (microkernel,
        CUDA events): separate multiplies and adds, or fused multiply-adds
        counted as two operations."""
        v = C.c_double()
        self._check(self.lib.rp3dg_measure_fp32_peak(self.device, int(bool(fused)), C.byref(v)))
        return v.value

    def narrowphase_device(self, algo, pairs, out, clip=True):
        """Asynchronous on the context stream, ordered after torch's current
        stream and before later work on it; pairs/out are DevicePairs/DeviceContacts."""
        pb, cb = pairs.struct(), out.struct()
        self.order_in()
        self._check(self.lib.rp3dg_narrowphase_device(self.h, int(algo), C.byref(pb), C.byref(cb), int(clip)))
        self.order_out()
        return out


MLP_NPARAMS = 6800
MLP_FEATURES = 24
MLP_CLASSES = 16


class AxisMLP:
    """The learned separating-axis proposal of a Context (device-side model)."""

    def __init__(self, ctx, seed=0):
        self.ctx = ctx
        ctx._check(ctx.lib.rp3dg_axis_mlp_init(ctx.h, int(seed)))

    def params(self):
        p = np.zeros(MLP_NPARAMS, np.float32)
        self.ctx._check(self.ctx.lib.rp3dg_axis_mlp_get_params(self.ctx.h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == MLP_NPARAMS
        self.ctx._check(self.ctx.lib.rp3dg_axis_mlp_set_params(self.ctx.h, p.ctypes.data))

    def features(self, dpairs):
        import torch
        f = torch.empty((dpairs.n, MLP_FEATURES), dtype=torch.float32, device=dpairs.shape1.device)
        pb = dpairs.struct()
        self.ctx.order_in()
        self.ctx._check(self.ctx.lib.rp3dg_axis_features(self.ctx.h, C.byref(pb), f.data_ptr()))
        self.ctx.order_out()
        return f

    def labels(self, dpairs, dcontacts):
        """Classes from the outcome of a fresh full-SAT pass over dpairs (its cache and flags)."""
        import torch
        y = torch.empty(dpairs.n, dtype=torch.uint8, device=dpairs.shape1.device)
        pb = dpairs.struct()
        self.ctx.order_in()
        self.ctx._check(self.ctx.lib.rp3dg_axis_labels(self.ctx.h, C.byref(pb), dcontacts.is_colliding.data_ptr(),
                                                       y.data_ptr()))
        self.ctx.order_out()
        return y

    def grads(self, x, y):
        import torch
        g = torch.empty(MLP_NPARAMS, dtype=torch.float32, device=x.device)
        loss = C.c_float()
        self.ctx.order_in()
        self.ctx._check(self.ctx.lib.rp3dg_axis_mlp_grads(self.ctx.h, x.data_ptr(), y.data_ptr(), int(x.shape[0]),
                                                          g.data_ptr(), C.addressof(loss)))
        self.ctx.order_out()
        return g, loss.value

    def train_step(self, x, y, lr=1e-3, want_loss=False):
        loss = C.c_float()
        self.ctx.order_in()
        self.ctx._check(self.ctx.lib.rp3dg_axis_mlp_train_step(self.ctx.h, x.data_ptr(), y.data_ptr(), int(x.shape[0]),
                                                               float(lr), C.addressof(loss) if want_loss else None))
        self.ctx.order_out()
        return loss.value if want_loss else None

    def predict(self, x):
        import torch
        c = torch.empty(x.shape[0], dtype=torch.uint8, device=x.device)
        self.ctx.order_in()
        self.ctx._check(self.ctx.lib.rp3dg_axis_mlp_predict(self.ctx.h, x.data_ptr(), int(x.shape[0]), c.data_ptr()))
        self.ctx.order_out()
        return c

    def enable(self, on=True):
        self.ctx._check(self.ctx.lib.rp3dg_set_learned_axis(self.ctx.h, int(on)))

    def stats(self, clear=True):
        t, c = C.c_uint64(), C.c_uint64()
        self.ctx._check(self.ctx.lib.rp3dg_learned_axis_stats(self.ctx.h, C.byref(t), C.byref(c), int(clear)))
        return t.value, c.value


def train_axis_mlp(ctx, mlp, x, y, epochs=4, batch=8192, lr=2e-3, seed=0, log=None):
    """Minibatch Adam over device tensors x (n x 24) and y (n); returns the
    per-epoch mean losses.  Shuffling uses a seeded permutation."""
    import torch
    n = int(x.shape[0])
    gen = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen).to(x.device)
        xs, ys = x[perm].contiguous(), y[perm].contiguous()
        tot, cnt = 0.0, 0
        for b0 in range(0, n - batch + 1, batch):
            want = (b0 // batch) % 16 == 0
            l = mlp.train_step(xs[b0:b0 + batch], ys[b0:b0 + batch], lr=lr, want_loss=want)
            if want:
                tot += l
                cnt += 1
        losses.append(tot / max(cnt, 1))
        if log:
            log(f"epoch {ep}: loss {losses[-1]:.4f}")
    return losses


class World:
    """A physics world stepped on the GPU (rp3dg_world_*): the drop-in for
    PhysicsWorld::update.  `scene` is a scenes.WorldScene; the context's shape
    table is replaced by the scene's."""

    def __init__(self, ctx, scene, threads=None):
        self.ctx, self.lib = ctx, ctx.lib
        ctx.set_shapes(ctx.scene_shapes(scene))
        self.nb = len(scene.bodies)
        self._keep = (np.ascontiguousarray(scene.settings).copy(), np.ascontiguousarray(scene.bodies),
                      np.ascontiguousarray(scene.colliders))
        st, bd, cd = self._keep
        h = C.c_void_p()
        rc = self.lib.rp3dg_world_create(ctx.h, st.ctypes.data, bd.ctypes.data, len(bd), cd.ctypes.data, len(cd),
                                         C.byref(h))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(ctx.h).decode())
        self.h = h
        self.set_threads(threads or (os.cpu_count() or 1))
        if getattr(scene, "joints", None) is not None and len(scene.joints):
            self.add_joints(scene.joints)

    def close(self):
        if self.h:
            self.lib.rp3dg_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_joints(self, joints, world=None):
        """createJoint for each row of `joints` (A.JOINT_DESC_DTYPE), before the first update."""
        j = np.ascontiguousarray(joints)
        if world is None:
            rc = self.lib.rp3dg_world_add_joints(self.h, j.ctypes.data, len(j))
        else:
            rc = self.lib.rp3dg_world_group_add_joints(self.h, int(world), j.ctypes.data, len(j))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())

    def contact_events(self, world=0):
        """EventListener::onContact of the last update: (events
        A.CONTACT_EVENT_DTYPE, normal + depth (n, 4), local points 1, local
        points 2)."""
        ne, npt = C.c_uint32(), C.c_uint32()
        rc = self.lib.rp3dg_world_get_contact_events(self.h, int(world), None, 0, None, None, None, 0,
                                                     C.byref(ne), C.byref(npt))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        ev = np.zeros(ne.value, A.CONTACT_EVENT_DTYPE)
        nd, l1, l2 = (np.zeros((npt.value, 4), np.float32) for _ in range(3))
        rc = self.lib.rp3dg_world_get_contact_events(self.h, int(world), ev.ctypes.data, len(ev), nd.ctypes.data,
                                                     l1.ctypes.data, l2.ctypes.data, len(nd), C.byref(ne),
                                                     C.byref(npt))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        return ev, nd, l1, l2

    def trigger_events(self, world=0):
        """The trigger events of the last update (structured array of
        A.CONTACT_EVENT_DTYPE, no points)."""
        n = C.c_uint32()
        rc = self.lib.rp3dg_world_get_trigger_events(self.h, int(world), None, 0, C.byref(n))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        ev = np.zeros(n.value, A.CONTACT_EVENT_DTYPE)
        rc = self.lib.rp3dg_world_get_trigger_events(self.h, int(world), ev.ctypes.data if len(ev) else None, len(ev),
                                                     C.byref(n))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        return ev

    def set_debug_rendering(self, items=A.DEBUG_ALL):
        """PhysicsWorld::setIsDebugRenderingEnabled(items != 0) with the
        DebugRenderer items of `items` (A.DEBUG_* bits) displayed."""
        rc = self.lib.rp3dg_world_set_debug_rendering(self.h, int(items))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())

    def set_body_debug(self, body=-1, enabled=True, world=0):
        """Body::setIsDebugEnabled for one body, or every body (body < 0)."""
        rc = self.lib.rp3dg_world_set_body_debug(self.h, int(world), int(body), int(bool(enabled)))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())

    def debug_primitives(self, world=0):
        """DebugRenderer's lines and triangles after the last update
        (structured arrays of A.DEBUG_LINE_DTYPE / A.DEBUG_TRIANGLE_DTYPE)."""
        nl, nt = C.c_uint32(), C.c_uint32()
        rc = self.lib.rp3dg_world_get_debug_primitives(self.h, int(world), None, 0, None, 0, C.byref(nl), C.byref(nt), 0)
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        lines = np.zeros(nl.value, A.DEBUG_LINE_DTYPE)
        tris = np.zeros(nt.value, A.DEBUG_TRIANGLE_DTYPE)
        rc = self.lib.rp3dg_world_get_debug_primitives(self.h, int(world), lines.ctypes.data if len(lines) else None,
                                                       len(lines), tris.ctypes.data if len(tris) else None, len(tris),
                                                       C.byref(nl), C.byref(nt), 0)
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        return lines, tris

    def raycast(self, rays, mode=A.RAYCAST_CLOSEST, max_hits=1, world=0):
        """PhysicsWorld::raycast for each row of `rays` (A.RAY_DTYPE) with the
        CLOSEST / ANY / ALL callback: (hits (n, max_hits) A.RAYCAST_HIT_DTYPE,
        hit counts (n,))."""
        r = np.ascontiguousarray(rays, dtype=A.RAY_DTYPE)
        n = len(r)
        hits = np.zeros((n, max_hits), A.RAYCAST_HIT_DTYPE)
        counts = np.zeros(n, np.uint32)
        rc = self.lib.rp3dg_world_raycast(self.h, int(world), r.ctypes.data, n, int(mode), int(max_hits),
                                          hits.ctypes.data, counts.ctypes.data)
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        return hits, counts

    def raycast_device(self, rays_ptr, n, hits_ptr, counts_ptr, mode=A.RAYCAST_CLOSEST, max_hits=1, world=0):
        """The raycast on device arrays (raw pointers); returns the traversal
        kernel's duration in ms."""
        ms = C.c_float()
        rc = self.lib.rp3dg_world_raycast_device(self.h, int(world), rays_ptr, int(n), int(mode), int(max_hits),
                                                 hits_ptr, counts_ptr, C.byref(ms))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        return ms.value

    def set_motor_speed(self, joint, speed, world=0):
        """HingeJoint / SliderJoint::setMotorSpeed on joint `joint` (creation
        order) of world `world`; a changed speed wakes the joint's bodies."""
        rc = self.lib.rp3dg_world_set_motor_speed(self.h, int(world), int(joint), float(speed))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())

    def update(self, dt=1.0 / 60.0, n=1):
        for _ in range(n):
            rc = self.lib.rp3dg_world_update(self.h, dt)
            if rc != 0:
                raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())

    def bodies(self):
        """(position (n,3), orientation (n,4), linear velocity, angular velocity, sleeping) in creation order."""
        n = self.nb
        p, q = np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32)
        lv, av = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
        sl = np.zeros(n, np.uint8)
        rc = self.lib.rp3dg_world_get_bodies(self.h, p.ctypes.data, q.ctypes.data, lv.ctypes.data, av.ctypes.data,
                                             sl.ctypes.data)
        assert rc == 0, rc
        return p, q, lv, av, sl

    def pairs(self):
        """Overlapping-pair ids in the reference's array order (enabled, then disabled)."""
        n = C.c_uint32()
        self.lib.rp3dg_world_get_pairs(self.h, None, 0, C.byref(n))
        out = np.zeros(n.value, np.uint64)
        self.lib.rp3dg_world_get_pairs(self.h, out.ctypes.data, n.value, C.byref(n))
        return out

    def contacts(self):
        """Manifolds of the last step in solver order: body1, body2, point
        counts, and per point normal|depth, local1, local2 (float4)."""
        nm, npt = C.c_uint32(), C.c_uint32()
        self.lib.rp3dg_world_get_contacts(self.h, None, None, None, 0, None, None, None, 0, C.byref(nm), C.byref(npt))
        b1, b2 = np.zeros(nm.value, np.int32), np.zeros(nm.value, np.int32)
        k = np.zeros(nm.value, np.uint8)
        nd, l1, l2 = (np.zeros((npt.value, 4), np.float32) for _ in range(3))
        rc = self.lib.rp3dg_world_get_contacts(self.h, b1.ctypes.data, b2.ctypes.data, k.ctypes.data, nm.value,
                                               nd.ctypes.data, l1.ctypes.data, l2.ctypes.data, npt.value,
                                               C.byref(nm), C.byref(npt))
        assert rc == 0, rc
        return b1, b2, k, nd, l1, l2

    PHASES = ("broadphase", "middle", "narrow", "islands", "pack", "dynamics", "colliders", "sleeping",
              "m.pool", "m.resets", "m.rows", "m.tables", "m.items", "b.queries", "b.remove", "b.items")

    def set_threads(self, n):
        """Host threads of the world's bookkeeping (results do not depend on it)."""
        rc = self.lib.rp3dg_world_set_threads(self.h, int(n))
        if rc != 0:
            raise Rp3dgError(rc, "bad thread count")

    def autotune(self, rounds=2):
        """Tune the island scheduling over the next 9 * rounds steps (results unchanged)."""
        rc = self.lib.rp3dg_world_autotune(self.h, int(rounds))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())

    def tuning(self):
        t = np.zeros(4, np.uint32)
        self.lib.rp3dg_world_get_tuning(self.h, t.ctypes.data)
        return {"small_max": int(t[0]), "giant_min": int(t[1]), "large_per_sm": int(t[2]), "tuning": bool(t[3])}

    def set_device_trees(self, enable=True):
        """Keep the worlds' broad-phase trees on the device (reinsertions and
        queries on the GPU) or on the host; results are identical."""
        rc = self.lib.rp3dg_world_set_device_trees(self.h, int(bool(enable)))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())

    @property
    def device_trees(self):
        v = C.c_int(0)
        self.lib.rp3dg_world_get_device_trees(self.h, C.byref(v))
        return bool(v.value)

    def set_solver(self, solver=SOLVER_EXACT, stats=False):
        """RP3DG_SOLVER_EXACT (the drop-in) or RP3DG_SOLVER_GRAPH_COLORED; with
        stats, every step records the solver statistics."""
        rc = self.lib.rp3dg_world_set_solver(self.h, int(solver), int(bool(stats)))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())

    def solver_stats(self):
        """The last step's solver statistics as a dict."""
        st = SolverStats()
        rc = self.lib.rp3dg_world_get_solver_stats(self.h, C.byref(st))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(self.ctx.h).decode())
        return {f: getattr(st, f) for f, _ in SolverStats._fields_ if f != "reserved"}

    def set_profiling(self, on=True):
        self.lib.rp3dg_world_set_profiling(self.h, int(on))

    def phase_times(self):
        t = np.zeros(16, np.float64)
        self.lib.rp3dg_world_get_phase_times(self.h, t.ctypes.data, 16)
        return {k: v for k, v in zip(self.PHASES, t.tolist()) if v or not k.startswith("m.")}

    def stats(self):
        s = np.zeros(1, A.WORLD_STATS_DTYPE)
        self.lib.rp3dg_world_get_stats(self.h, s.ctypes.data)
        return {k: int(s[k][0]) for k in A.WORLD_STATS_DTYPE.names if k != "reserved"}


class WorldGroup(World):
    """Many independent worlds stepped together (rp3dg_world_group_*).  All
    scenes must share one shape table (scenes.merge_shapes builds it); world k
    is then read with bodies(k) / pairs(k) / contacts(k)."""

    def __init__(self, ctx, scenes_, shapes, threads=None):
        self.ctx, self.lib = ctx, ctx.lib
        if any(getattr(s, "heightfields", None) or getattr(s, "convex_meshes", None) or
               getattr(s, "concave_meshes", None) for s in scenes_):
            # the table is the scenes' tables back to back (scenes.merge_shapes):
            # each segment gets its scene's height fields and convex meshes
            shapes = np.array(shapes, copy=True)
            base = 0
            for s in scenes_:
                seg = ctx.scene_shapes(s)
                shapes[base:base + len(seg)] = seg
                base += len(seg)
            if base != len(shapes):
                raise ValueError("height fields or convex meshes need the table of scenes.merge_shapes")
        ctx.set_shapes(shapes)
        threads = threads or (os.cpu_count() or 1)
        bodies = np.concatenate([s.bodies for s in scenes_])
        colliders = np.concatenate([s.colliders for s in scenes_])
        boff = np.concatenate([[0], np.cumsum([len(s.bodies) for s in scenes_])]).astype(np.uint32)
        coff = np.concatenate([[0], np.cumsum([len(s.colliders) for s in scenes_])]).astype(np.uint32)
        self.sizes = [len(s.bodies) for s in scenes_]
        self.nb = int(boff[-1])
        self._keep = (np.ascontiguousarray(scenes_[0].settings).copy(), bodies, colliders, boff, coff)
        st = self._keep[0]
        h = C.c_void_p()
        rc = self.lib.rp3dg_world_group_create(ctx.h, st.ctypes.data, len(scenes_), boff.ctypes.data, bodies.ctypes.data,
                                               coff.ctypes.data, colliders.ctypes.data, int(threads), C.byref(h))
        if rc != 0:
            raise Rp3dgError(rc, self.lib.rp3dg_last_error(ctx.h).decode())
        self.h = h
        for k, sc in enumerate(scenes_):
            if getattr(sc, "joints", None) is not None and len(sc.joints):
                self.add_joints(sc.joints, world=k)

    def bodies(self, world=None):
        if world is None:
            return super().bodies()
        n = self.sizes[world]
        p, q = np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32)
        lv, av = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
        sl = np.zeros(n, np.uint8)
        rc = self.lib.rp3dg_world_group_get_bodies(self.h, world, p.ctypes.data, q.ctypes.data, lv.ctypes.data,
                                                   av.ctypes.data, sl.ctypes.data)
        assert rc == 0, rc
        return p, q, lv, av, sl

    def pairs(self, world=0):
        n = C.c_uint32()
        self.lib.rp3dg_world_group_get_pairs(self.h, world, None, 0, C.byref(n))
        out = np.zeros(n.value, np.uint64)
        self.lib.rp3dg_world_group_get_pairs(self.h, world, out.ctypes.data, n.value, C.byref(n))
        return out

    def contacts(self, world=0):
        nm, npt = C.c_uint32(), C.c_uint32()
        self.lib.rp3dg_world_group_get_contacts(self.h, world, None, None, None, 0, None, None, None, 0,
                                                C.byref(nm), C.byref(npt))
        b1, b2 = np.zeros(nm.value, np.int32), np.zeros(nm.value, np.int32)
        k = np.zeros(nm.value, np.uint8)
        nd, l1, l2 = (np.zeros((npt.value, 4), np.float32) for _ in range(3))
        rc = self.lib.rp3dg_world_group_get_contacts(self.h, world, b1.ctypes.data, b2.ctypes.data, k.ctypes.data,
                                                     nm.value, nd.ctypes.data, l1.ctypes.data, l2.ctypes.data,
                                                     npt.value, C.byref(nm), C.byref(npt))
        assert rc == 0, rc
        return b1, b2, k, nd, l1, l2
