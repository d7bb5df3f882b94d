// Test infrastructure, not product code: a thin C driver linked against the
// reference engine (ReactPhysics3D v0.10.2) built from its own sources by
// oracle/Makefile.  It fills the reference's own NarrowPhaseInfoBatch from the
// struct-of-arrays batches declared in include/rp3dg.h, runs the reference's
// algorithm objects on them (the "alternative harness": algorithm objects
// called directly, batchStartIndex always 0), and copies the results back
// into the same SoA layout, so the CUDA library, the C restatement and the
// reference itself can be compared value for value.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// the resulting oracle/_ref/librp3d_ref_*.so.
// The manifold-reduction entry below calls two private members of
// CollisionDetectionSystem directly: this translation unit is compiled with
// -fno-access-control (oracle/Makefile), which lifts access checks without
// changing any class layout; the reference objects are compiled unchanged.
#include <algorithm>
#include <array>
#include <atomic>
#include <functional>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <reactphysics3d/reactphysics3d.h>
#include <reactphysics3d/collision/narrowphase/NarrowPhaseInfoBatch.h>
#include <reactphysics3d/collision/narrowphase/SphereVsSphereAlgorithm.h>
#include <reactphysics3d/collision/narrowphase/SphereVsCapsuleAlgorithm.h>
#include <reactphysics3d/collision/narrowphase/CapsuleVsCapsuleAlgorithm.h>
#include <reactphysics3d/collision/narrowphase/SphereVsConvexPolyhedronAlgorithm.h>
#include <reactphysics3d/collision/narrowphase/CapsuleVsConvexPolyhedronAlgorithm.h>
#include <reactphysics3d/collision/narrowphase/ConvexPolyhedronVsConvexPolyhedronAlgorithm.h>
#include <reactphysics3d/collision/ContactPointInfo.h>
#include <reactphysics3d/engine/OverlappingPairs.h>
#include <reactphysics3d/memory/DefaultAllocator.h>

#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "../include/rp3dg.h"

using namespace reactphysics3d;

namespace {

struct MeshRec {
    std::vector<float> vertices;          // nv*3
    std::vector<uint32_t> indices;        // concatenated face indices
    std::vector<PolygonVertexArray::PolygonFace> faces;
    std::unique_ptr<PolygonVertexArray> pva;
    ConvexMesh* mesh = nullptr;
};

struct Harness {
    PhysicsCommon common;
    std::vector<std::unique_ptr<MeshRec>> meshes;
    std::vector<ConvexMeshShape*> instances;
};

Harness* g_h = nullptr;

Harness& H() {
    if (!g_h) g_h = new Harness();
    return *g_h;
}

// Shapes created for one narrowphase call.  The reference keeps raw
// CollisionShape pointers in each NarrowPhaseInfo (NarrowPhaseInfoBatch.h:82-85).
std::vector<CollisionShape*> make_shapes(const rp3dg_shape* shapes, uint32_t nb) {
    Harness& h = H();
    std::vector<CollisionShape*> out(nb, nullptr);
    for (uint32_t i = 0; i < nb; i++) {
        const rp3dg_shape& s = shapes[i];
        switch (s.kind) {
            case RP3DG_SHAPE_SPHERE: out[i] = h.common.createSphereShape(s.params[0]); break;
            // createCapsuleShape(radius, height) with height = 2 * halfHeight
            case RP3DG_SHAPE_CAPSULE: out[i] = h.common.createCapsuleShape(s.params[0], s.params[1] + s.params[1]); break;
            case RP3DG_SHAPE_BOX: out[i] = h.common.createBoxShape(Vector3(s.params[0], s.params[1], s.params[2])); break;
            case RP3DG_SHAPE_CONVEX_MESH: out[i] = h.instances.at(s.mesh); break;
            default: out[i] = nullptr;
        }
    }
    return out;
}

void destroy_shapes(const rp3dg_shape* shapes, std::vector<CollisionShape*>& v) {
    Harness& h = H();
    for (size_t i = 0; i < v.size(); i++) {
        if (!v[i]) continue;
        switch (shapes[i].kind) {
            case RP3DG_SHAPE_SPHERE: h.common.destroySphereShape(static_cast<SphereShape*>(v[i])); break;
            case RP3DG_SHAPE_CAPSULE: h.common.destroyCapsuleShape(static_cast<CapsuleShape*>(v[i])); break;
            case RP3DG_SHAPE_BOX: h.common.destroyBoxShape(static_cast<BoxShape*>(v[i])); break;
            default: break;
        }
    }
}

LastFrameCollisionInfo unpack_cache(const rp3dg_lastframe& c) {
    LastFrameCollisionInfo l;
    l.gjkSeparatingAxis = Vector3(c.gjk_axis[0], c.gjk_axis[1], c.gjk_axis[2]);
    l.isValid = (c.flags & RP3DG_LF_IS_VALID) != 0;
    l.isObsolete = (c.flags & RP3DG_LF_IS_OBSOLETE) != 0;
    l.wasColliding = (c.flags & RP3DG_LF_WAS_COLLIDING) != 0;
    l.wasUsingGJK = (c.flags & RP3DG_LF_WAS_USING_GJK) != 0;
    l.wasUsingSAT = (c.flags & RP3DG_LF_WAS_USING_SAT) != 0;
    l.satIsAxisFacePolyhedron1 = (c.flags & RP3DG_LF_SAT_FACE_POLY1) != 0;
    l.satIsAxisFacePolyhedron2 = (c.flags & RP3DG_LF_SAT_FACE_POLY2) != 0;
    l.satMinAxisFaceIndex = c.sat_face;
    l.satMinEdge1Index = c.sat_edge1;
    l.satMinEdge2Index = c.sat_edge2;
    return l;
}

void pack_cache(const LastFrameCollisionInfo& l, rp3dg_lastframe& c) {
    c.gjk_axis[0] = float(l.gjkSeparatingAxis.x);
    c.gjk_axis[1] = float(l.gjkSeparatingAxis.y);
    c.gjk_axis[2] = float(l.gjkSeparatingAxis.z);
    uint8_t f = 0;
    if (l.isValid) f |= RP3DG_LF_IS_VALID;
    if (l.isObsolete) f |= RP3DG_LF_IS_OBSOLETE;
    if (l.wasColliding) f |= RP3DG_LF_WAS_COLLIDING;
    if (l.wasUsingGJK) f |= RP3DG_LF_WAS_USING_GJK;
    if (l.wasUsingSAT) f |= RP3DG_LF_WAS_USING_SAT;
    if (l.satIsAxisFacePolyhedron1) f |= RP3DG_LF_SAT_FACE_POLY1;
    if (l.satIsAxisFacePolyhedron2) f |= RP3DG_LF_SAT_FACE_POLY2;
    c.flags = f;
    c.sat_face = l.satMinAxisFaceIndex;
    c.sat_edge1 = l.satMinEdge1Index;
    c.sat_edge2 = l.satMinEdge2Index;
}

// One slice of a batch: its own allocator, NarrowPhaseInfoBatch and caches.
struct Slice {
    uint32_t begin = 0, end = 0;
    double seconds = 0.0;
    bool any = false;
};

bool run_algorithm(int algorithm, NarrowPhaseInfoBatch& batch, uint32_t n, bool clip, MemoryAllocator& alloc) {
    switch (algorithm) {
        case RP3DG_ALGO_SPHERE_VS_SPHERE: { SphereVsSphereAlgorithm a; return a.testCollision(batch, 0, n, alloc); }
        case RP3DG_ALGO_SPHERE_VS_CAPSULE: { SphereVsCapsuleAlgorithm a; return a.testCollision(batch, 0, n, alloc); }
        case RP3DG_ALGO_CAPSULE_VS_CAPSULE: { CapsuleVsCapsuleAlgorithm a; return a.testCollision(batch, 0, n, alloc); }
        case RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON: { SphereVsConvexPolyhedronAlgorithm a; return a.testCollision(batch, 0, n, clip, alloc); }
        case RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON: { CapsuleVsConvexPolyhedronAlgorithm a; return a.testCollision(batch, 0, n, clip, alloc); }
        case RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON: { ConvexPolyhedronVsConvexPolyhedronAlgorithm a; return a.testCollision(batch, 0, n, clip, alloc); }
    }
    return false;
}

void run_slice(int algorithm, const std::vector<CollisionShape*>& shp, const rp3dg_pair_batch* p,
               const rp3dg_contact_batch* out, bool clip, int repeats, Slice& s) {
    DefaultAllocator alloc;
    // The batch only stores a reference to the overlapping pairs and never
    // touches it (NarrowPhaseInfoBatch.cpp:35-38), so any storage will do.
    alignas(64) static thread_local unsigned char fake_pairs[sizeof(void*) * 4];
    OverlappingPairs& pairs = *reinterpret_cast<OverlappingPairs*>(fake_pairs);
    const uint32_t n = s.end - s.begin;
    std::vector<LastFrameCollisionInfo> caches(n);
    double best = 1e300;
    for (int rep = 0; rep < repeats; rep++) {
        NarrowPhaseInfoBatch batch(pairs, alloc);
        batch.narrowPhaseInfos.reserve(n);
        for (uint32_t k = 0; k < n; k++) {
            const uint32_t i = s.begin + k;
            caches[k] = p->cache ? unpack_cache(p->cache[i]) : LastFrameCollisionInfo();
            const Transform t1(Vector3(p->pos1[i].x, p->pos1[i].y, p->pos1[i].z),
                               Quaternion(p->rot1[i].x, p->rot1[i].y, p->rot1[i].z, p->rot1[i].w));
            const Transform t2(Vector3(p->pos2[i].x, p->pos2[i].y, p->pos2[i].z),
                               Quaternion(p->rot2[i].x, p->rot2[i].y, p->rot2[i].z, p->rot2[i].w));
            const bool report = p->report_contacts ? p->report_contacts[i] != 0 : true;
            batch.addNarrowPhaseInfo(i, Entity(2 * i, 0), Entity(2 * i + 1, 0), shp[p->shape1[i]], shp[p->shape2[i]],
                                     t1, t2, report, &caches[k], alloc);
        }
        auto t0 = std::chrono::steady_clock::now();
        s.any = run_algorithm(algorithm, batch, n, clip, alloc);
        auto t1 = std::chrono::steady_clock::now();
        best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
        if (rep + 1 == repeats && out) {
            for (uint32_t k = 0; k < n; k++) {
                const uint32_t i = s.begin + k;
                auto& info = batch.narrowPhaseInfos[k];
                out->is_colliding[i] = info.isColliding ? 1 : 0;
                const uint32_t nc = std::min<uint32_t>(info.nbContactPoints, out->max_contacts);
                out->nb_contacts[i] = uint8_t(nc);
                for (uint32_t c = 0; c < nc; c++) {
                    const ContactPointInfo& cp = info.contactPoints[c];
                    const size_t o = size_t(c) * p->n + i;
                    out->normal_depth[o] = {float(cp.normal.x), float(cp.normal.y), float(cp.normal.z), float(cp.penetrationDepth)};
                    out->local1[o] = {float(cp.localPoint1.x), float(cp.localPoint1.y), float(cp.localPoint1.z), 0.f};
                    out->local2[o] = {float(cp.localPoint2.x), float(cp.localPoint2.y), float(cp.localPoint2.z), 0.f};
                }
                if (p->cache) pack_cache(caches[k], p->cache[i]);
            }
        }
        // Contact points must be reset before the batch is cleared (assert in
        // NarrowPhaseInfoBatch::clear, NarrowPhaseInfoBatch.cpp:59).
        for (uint32_t k = 0; k < n; k++) batch.resetContactPoints(k);
    }
    s.seconds = best;
}

}  // namespace

extern "C" {

// Precision of this build: 4 = float, 8 = double.
int ref_decimal_size() { return int(sizeof(decimal)); }

// Convex mesh from polygon faces (PhysicsCommon::createConvexMesh(PolygonVertexArray)).
int ref_create_convex_mesh(const float* vertices, uint32_t nv, const uint32_t* face_indices,
                           const uint32_t* face_sizes, uint32_t nf, int32_t* mesh_id) {
    Harness& h = H();
    auto m = std::make_unique<MeshRec>();
    m->vertices.assign(vertices, vertices + 3 * nv);
    uint32_t total = 0;
    for (uint32_t f = 0; f < nf; f++) {
        PolygonVertexArray::PolygonFace pf;
        pf.nbVertices = face_sizes[f];
        pf.indexBase = total;
        m->faces.push_back(pf);
        total += face_sizes[f];
    }
    m->indices.assign(face_indices, face_indices + total);
    m->pva = std::make_unique<PolygonVertexArray>(nv, m->vertices.data(), 3 * sizeof(float), m->indices.data(),
                                                  sizeof(uint32_t), nf, m->faces.data(),
                                                  PolygonVertexArray::VertexDataType::VERTEX_FLOAT_TYPE,
                                                  PolygonVertexArray::IndexDataType::INDEX_INTEGER_TYPE);
    std::vector<Message> msgs;
    m->mesh = h.common.createConvexMesh(*m->pva, msgs);
    if (!m->mesh) return -1;
    h.meshes.push_back(std::move(m));
    *mesh_id = int32_t(h.meshes.size() - 1);
    return 0;
}

int ref_create_convex_mesh_shape(int32_t mesh_id, float sx, float sy, float sz, int32_t* instance_id) {
    Harness& h = H();
    if (mesh_id < 0 || size_t(mesh_id) >= h.meshes.size()) return -1;
    h.instances.push_back(h.common.createConvexMeshShape(h.meshes[mesh_id]->mesh, Vector3(sx, sy, sz)));
    *instance_id = int32_t(h.instances.size() - 1);
    return 0;
}

// Tables of a convex mesh shape instance (same layout as rp3dg_get_convex_mesh_tables).
int ref_get_convex_mesh_tables(int32_t instance_id, uint32_t* nb_vertices, uint32_t* nb_faces,
                               uint32_t* nb_half_edges, uint32_t* half_edges, float* face_normals,
                               uint32_t* face_edge, float* centroid, float* vertices,
                               uint32_t cap_he, uint32_t cap_faces) {
    Harness& h = H();
    if (instance_id < 0 || size_t(instance_id) >= h.instances.size()) return -1;
    const ConvexMeshShape* s = h.instances[instance_id];
    *nb_vertices = s->getNbVertices();
    *nb_faces = s->getNbFaces();
    *nb_half_edges = s->getNbHalfEdges();
    if (*nb_half_edges > cap_he || *nb_faces > cap_faces) return -2;
    for (uint32_t e = 0; e < *nb_half_edges; e++) {
        const HalfEdgeStructure::Edge& ed = s->getHalfEdge(e);
        half_edges[4 * e + 0] = ed.vertexIndex;
        half_edges[4 * e + 1] = ed.twinEdgeIndex;
        half_edges[4 * e + 2] = ed.faceIndex;
        half_edges[4 * e + 3] = ed.nextEdgeIndex;
    }
    for (uint32_t f = 0; f < *nb_faces; f++) {
        const Vector3 nrm = s->getFaceNormal(f);
        face_normals[3 * f + 0] = float(nrm.x);
        face_normals[3 * f + 1] = float(nrm.y);
        face_normals[3 * f + 2] = float(nrm.z);
        face_edge[f] = s->getFace(f).edgeIndex;
    }
    const Vector3 c = s->getCentroid();
    centroid[0] = float(c.x); centroid[1] = float(c.y); centroid[2] = float(c.z);
    if (vertices) {
        for (uint32_t v = 0; v < *nb_vertices; v++) {
            const Vector3 p = s->getVertexPosition(v);
            vertices[3 * v + 0] = float(p.x); vertices[3 * v + 1] = float(p.y); vertices[3 * v + 2] = float(p.z);
        }
    }
    return 0;
}

// Convex hull of a point cloud through the reference's QuickHull
// (PhysicsCommon::createConvexMesh(const VertexArray&), PhysicsCommon.cpp:638-648).
// Writes the hull's vertices and polygon faces.
int ref_quickhull(const float* points, uint32_t np, float* out_vertices, uint32_t cap_vertices,
                  uint32_t* out_nv, uint32_t* out_face_indices, uint32_t cap_indices,
                  uint32_t* out_face_sizes, uint32_t cap_faces, uint32_t* out_nf) {
    Harness& h = H();
    VertexArray va(points, 3 * sizeof(float), np, VertexArray::DataType::VERTEX_FLOAT_TYPE);
    std::vector<Message> msgs;
    ConvexMesh* mesh = h.common.createConvexMesh(va, msgs);
    if (!mesh) return -1;
    const HalfEdgeStructure& hes = mesh->getHalfEdgeStructure();
    const uint32_t nv = mesh->getNbVertices(), nf = hes.getNbFaces();
    if (nv > cap_vertices || nf > cap_faces) return -2;
    for (uint32_t v = 0; v < nv; v++) {
        const Vector3& p = mesh->getVertex(v);
        out_vertices[3 * v] = float(p.x); out_vertices[3 * v + 1] = float(p.y); out_vertices[3 * v + 2] = float(p.z);
    }
    uint32_t k = 0;
    for (uint32_t f = 0; f < nf; f++) {
        const auto& fv = hes.getFace(f).faceVertices;
        out_face_sizes[f] = uint32_t(fv.size());
        for (uint32_t j = 0; j < fv.size(); j++) {
            if (k >= cap_indices) return -2;
            out_face_indices[k++] = fv[j];
        }
    }
    *out_nv = nv;
    *out_nf = nf;
    h.common.destroyConvexMesh(mesh);
    return 0;
}

// Run one reference algorithm over a batch (host arrays, rp3dg.h layout).
// nthreads > 1 splits the batch into contiguous slices, one reference batch
// per thread (the engine itself is single-threaded; shapes are only read).
// repeats > 1 re-runs the timed testCollision call and keeps the best time.
// *seconds receives the wall time of the slowest slice's testCollision calls.
int ref_narrowphase(int algorithm, const rp3dg_shape* shapes, uint32_t nb_shapes, const rp3dg_pair_batch* pairs,
                    const rp3dg_contact_batch* out, int clip_with_previous_axis, int nthreads, int repeats,
                    double* seconds) {
    if (!pairs || algorithm < 1 || algorithm > 6) return -1;
    std::vector<CollisionShape*> shp = make_shapes(shapes, nb_shapes);
    const uint32_t n = pairs->n;
    if (nthreads < 1) nthreads = 1;
    if (repeats < 1) repeats = 1;
    std::vector<Slice> slices(nthreads);
    for (int t = 0; t < nthreads; t++) {
        slices[t].begin = uint32_t((uint64_t(n) * t) / nthreads);
        slices[t].end = uint32_t((uint64_t(n) * (t + 1)) / nthreads);
    }
    auto w0 = std::chrono::steady_clock::now();
    if (nthreads == 1) {
        run_slice(algorithm, shp, pairs, out, clip_with_previous_axis != 0, repeats, slices[0]);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nthreads; t++)
            th.emplace_back(run_slice, algorithm, std::cref(shp), pairs, out, clip_with_previous_axis != 0, repeats,
                            std::ref(slices[t]));
        for (auto& x : th) x.join();
    }
    auto w1 = std::chrono::steady_clock::now();
    (void)w0; (void)w1;
    double worst = 0.0;
    for (auto& s : slices) worst = std::max(worst, s.seconds);
    if (seconds) *seconds = worst;
    destroy_shapes(shapes, shp);
    return 0;
}

// Manifold of every colliding convex pair reduced by the reference's own
// CollisionDetectionSystem::reduceContactPoints (when it has more than 4
// points) and removeDuplicatedContactPointsInManifold, exactly as
// reducePotentialContactManifolds applies them (CollisionDetectionSystem.cpp:
// 1394-1458).  Same in/out convention as rp3do_reduce_contacts.
int ref_reduce_contacts(const rp3dg_pair_batch* p, const rp3dg_contact_batch* c, uint8_t* kept) {
    Harness& h = H();
    static PhysicsWorld* world = nullptr;
    if (!world) world = h.common.createPhysicsWorld();
    const CollisionDetectionSystem& cds = world->mCollisionDetection;
    DefaultAllocator alloc;
    const uint32_t n = p->n;
    for (uint32_t i = 0; i < n; i++) {
        if (p->cache) {
            // the two assignments of processPotentialContacts (:1209-1217) on the
            // reference's own LastFrameCollisionInfo
            LastFrameCollisionInfo l = unpack_cache(p->cache[i]);
            l.wasColliding = c->is_colliding[i] != 0;
            l.isValid = true;
            pack_cache(l, p->cache[i]);
        }
        uint32_t nb = c->nb_contacts[i];
        Array<ContactPointInfo> pts(alloc, 16);
        for (uint32_t k = 0; k < nb; k++) {
            const size_t o = size_t(k) * n + i;
            ContactPointInfo cp;
            cp.normal = Vector3(c->normal_depth[o].x, c->normal_depth[o].y, c->normal_depth[o].z);
            cp.penetrationDepth = c->normal_depth[o].w;
            cp.localPoint1 = Vector3(c->local1[o].x, c->local1[o].y, c->local1[o].z);
            cp.localPoint2 = Vector3(c->local2[o].x, c->local2[o].y, c->local2[o].z);
            pts.add(cp);
        }
        ContactManifoldInfo m(i);
        for (uint32_t k = 0; k < nb; k++) m.potentialContactPointsIndices[k] = k;
        m.nbPotentialContactPoints = uint8_t(nb);
        if (nb > 0 && c->is_colliding[i]) {
            const Transform t1(Vector3(p->pos1[i].x, p->pos1[i].y, p->pos1[i].z),
                               Quaternion(p->rot1[i].x, p->rot1[i].y, p->rot1[i].z, p->rot1[i].w));
            if (nb > 4) cds.reduceContactPoints(m, t1, pts);
            cds.removeDuplicatedContactPointsInManifold(m, pts);
        }
        const uint32_t mm = std::min<uint32_t>(m.nbPotentialContactPoints, 4);
        rp3dg_float4 nd[4], l1[4], l2[4];
        for (uint32_t k = 0; k < mm; k++) {
            const size_t o = size_t(m.potentialContactPointsIndices[k]) * n + i;
            nd[k] = c->normal_depth[o]; l1[k] = c->local1[o]; l2[k] = c->local2[o];
        }
        for (uint32_t k = 0; k < mm; k++) {
            const size_t o = size_t(k) * n + i;
            c->normal_depth[o] = nd[k]; c->local1[o] = l1[k]; c->local2[o] = l2[k];
        }
        if (kept) for (uint32_t k = 0; k < 4; k++) kept[4 * size_t(i) + k] = uint8_t(k < mm ? m.potentialContactPointsIndices[k] : 255);
        c->nb_contacts[i] = uint8_t(mm);
    }
    return 0;
}

}  // extern "C"
