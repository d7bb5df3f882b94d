// Layouts shared by the host runtime and the kernels.
#pragma once
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

// A height field (HeightField + HeightFieldShape scale) as the middle phase
// reads it: heights[y * ncol + x], unscaled local bounds, height origin.
struct HfDesc {
    uint32_t ncol, nrow;
    float width, length, origin;
    float bmin[3], bmax[3];
    float scale[3];
    const float* heights;  // device
};

}  // namespace rp3dg
