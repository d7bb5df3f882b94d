// Layouts shared by the host runtime and the kernels.
#pragma once
#include <vector_types.h>

#include <cstdint>

namespace rp3dg {

// Largest polygon a convex mesh face may have (clip buffers are sized from it).
constexpr uint32_t MAX_FACE_VERTICES = 16;
constexpr uint32_t CLIP_MAX = 2 * MAX_FACE_VERTICES;
// Largest mesh a kernel accepts (faces, half-edge and vertex indices fit uint8
// in the temporal-coherence cache exactly like the reference's uint8 fields).
constexpr uint32_t MAX_MESH_FACES = 256;
constexpr uint32_t MAX_MESH_HALF_EDGES = 256;
constexpr uint32_t MAX_MESH_VERTICES = 4096;

// One convex-mesh shape instance (mesh + scale) inside the device mesh arena.
// All offsets are in 32-bit words from the start of the arena.
struct MeshHdr {
    uint32_t nv, nf, nhe, pad0;
    uint32_t off_verts;       // nv * 3 floats, unscaled (used by the support search)
    uint32_t off_sverts;      // nv * 3 floats, vertex * scale
    uint32_t off_normals;     // nf * 3 floats, scaled unit normals
    uint32_t off_face_start;  // nf uint32: first index in face_verts
    uint32_t off_face_count;  // nf uint32
    uint32_t off_face_verts;  // sum(face_count) uint32
    uint32_t off_face_edge;   // nf uint32: Face::edgeIndex
    uint32_t off_edges;       // nhe * 4 uint32: vertex, twin, face, next
    float centroid[3];        // mesh centroid * scale
    uint32_t pad1;
};
static_assert(sizeof(MeshHdr) == 64, "MeshHdr layout");

// Box topology (PhysicsCommon::initBoxShapeHalfEdgeStructure).
// gauss[e] describes half-edge e for the Gauss-map test against a box:
//   [0] = k | (negD << 2):  edge vector v(e.vertex) - v(twin.vertex) lies on
//                           axis k, negative when negD is set
//   [1] = m | (negC << 2):  c = -normal(e.face) lies on axis m
//   [2] = n | (negD2 << 2): d = -normal(twin.face) lies on axis n
struct BoxTables {
    uint8_t edges[24][4];  // vertex, twin, face, next
    uint8_t face_verts[24];
    uint8_t face_edge[6];
    uint8_t pad[2];
    uint8_t gauss[24][4];
    uint8_t axis_edges[3][4];  // even half-edges along x, y, z (increasing index)
    // TriangleShape topology (PhysicsCommon::initTriangleShapeHalfEdgeStructure):
    // faces (0, 1, 2) and (0, 2, 1)
    uint8_t tri_edges[6][4];   // vertex, twin, face, next
    uint8_t tri_face_edge[2];
    uint8_t pad2[2];
};

// Steps of the reference's narrow-phase code paths, counted per batch by the
// event-counting build of the kernels (RP3DG_COUNT_EVENTS): each event is one
// execution of a fixed piece of the reference's arithmetic, so the FP32
// operations of a batch are the event counts times a static per-event op
// table.  The order is part of the C ABI (rp3dg_narrowphase_count_events).
enum NpEvent : uint32_t {
    EV_POLY_SETUP = 0,     // SAT polyhedron pair: both relative transforms (SATAlgorithm.cpp:502-503)
    EV_FACE_TEST,          // testSingleFaceDirectionPolyhedronVsPolyhedron without the support (:1087-1110)
    EV_SUPPORT_BOX,        // BoxShape::getLocalSupportPointWithoutMargin
    EV_SUPPORT_VERTEX,     // one vertex of ConvexMeshShape::getLocalSupportPointWithoutMargin
    EV_SUPPORT_TRI,        // TriangleShape::getLocalSupportPointWithoutMargin
    EV_SUPPORT_CAPSULE,    // CapsuleShape::getLocalSupportPointWithoutMargin
    EV_EDGE1,              // edge of polyhedron 1 in polyhedron-2 space (:749-755)
    EV_GAUSS,              // edge-2 direction + testEdgesBuildMinkowskiFace (:763-769, :1146-1191)
    EV_EDGE_DIST,          // centroid + computeDistanceBetweenEdges + comparisons (:771-809, :1040-1083)
    EV_CLIP_SETUP,         // computePolyhedronVsPolyhedronFaceContactPoints: axes (:921-928)
    EV_ANTIPARALLEL,       // one face of findMostAntiParallelFace (ConvexPolyhedronShape.h:105-123)
    EV_INC_VERTEX,         // incident face vertex into reference space (:945-948)
    EV_CLIP_PLANE,         // one reference-face side plane + clipPolygonWithPlane set-up (:958-965, mathematics_functions.h:339-343)
    EV_CLIP_VERTEX,        // one input vertex of clipPolygonWithPlane (mathematics_functions.h:346-392)
    EV_CLIP_INTERSECT,     // one computePlaneSegmentIntersection + interpolation
    EV_CLIP_DEPTH,         // depth of one clipped vertex (:1000-1002)
    EV_CONTACT,            // one face contact: incident point + projection (:1007-1013)
    EV_EDGE_CONTACT,       // edge-edge contact: closest points, transforms (:853-864)
    EV_GJK_SETUP,          // GJKAlgorithm::testCollision transforms (GJKAlgorithm.cpp:79-92)
    EV_GJK_ITER,           // one GJK iteration without supports and simplex (:118-190)
    EV_SX_SEG,             // VoronoiSimplex closest point, 2 points (VoronoiSimplex.cpp:304-331)
    EV_SX_TRI,             // 3 points (:336-451)
    EV_SX_TET,             // 4 points (:456-575)
    EV_GJK_CONTACT,        // GJK contact in margin (GJKAlgorithm.cpp:196-233)
    EV_SPHERE_FACE,        // one face of the SAT sphere test (SATAlgorithm.cpp:82-95, :147-162)
    EV_SPHERE_POLY_CONTACT,// SAT sphere contact (:100-140)
    EV_CAPSULE_FACE,       // one face of the SAT capsule test (:197-211, :357-376)
    EV_CAPSULE_EDGE,       // one edge of the SAT capsule test, Minkowski-face check (:218-236, :476-482)
    EV_CAPSULE_EDGE_AXIS,  // its edge vs inner-segment depth (:322-354)
    EV_CAPSULE_CLIP,       // one side plane of computeCapsulePolyhedronFaceContactPoints (:381-470)
    EV_CLOSED_FORM,        // sphere-sphere / sphere-capsule / capsule-capsule: one whole pair test
    EV_CLOSED_FORM_CONTACT,// ... and one of its contacts
    EV_CAPSULE_GJK_FACE,   // one face of the in-margin capsule face search (CapsuleVsConvexPolyhedronAlgorithm.cpp:104-160)
    EV_TRI_SMOOTH,         // one smooth-normal correction of a triangle contact (TriangleShape.h:309-365)
    NP_EVENT_USED,
    NP_EVENT_COUNT = 40    // slots of the C ABI array (the rest stay zero)
};

// A height field (HeightField + HeightFieldShape scale) as the middle phase
// reads it: heights[y * ncol + x], unscaled local bounds, height origin.
struct HfDesc {
    uint32_t ncol, nrow;
    float width, length, origin;
    float bmin[3], bmax[3];
    float scale[3];
    const float* heights;  // device
};

// One node of a DynamicAABBTree as the GPU traversals read it: lo = (AABB
// min, child 0), hi = (AABB max, child 1), the children as int bits (-1:
// none).  A leaf has child 0 = -2 - its data (collider or triangle index).
struct __align__(16) RayNode {
    float4 lo, hi;
};

// A concave mesh shape (ConcaveMeshShape over a TriangleMesh, with its
// scale) as the middle phase, the raycasts and the debug renderer read it.
struct CmDesc {
    uint32_t nv, nt;
    int32_t root;             // root node of the triangle tree (-1: empty)
    uint32_t mesh;            // the triangle mesh's id
    float scale[3];
    float inv_scale[3];       // decimal(1.0) / scale per axis
    const uint32_t* tris;     // device: 3 vertex indices per triangle
    const float* sverts;      // device: 3 floats per vertex, vertex * scale
    const float* snormals;    // device: 3 floats per vertex, scaled vertex normals
    const RayNode* nodes;     // device: the mesh's DynamicAABBTree over the unscaled triangles
};

}  // namespace rp3dg
