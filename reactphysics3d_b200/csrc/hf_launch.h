// Launch interface of the convex vs concave middle phase (heightfield.cu):
// height fields and concave triangle meshes.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"
#include "rp3dg_internal.h"

namespace rp3dg {

// One convex vs concave pair of the middle phase:
//   item = (convex collider row, concave collider row, height-field or
//           concave-mesh id, flags: bit 0 = shape 1 is the convex one)
constexpr int HF_SHAPE1_CONVEX = 1;
constexpr int HF_NO_REPORT = 2;   // a collider of the pair is a trigger: no contact points
constexpr int HF_MESH = 4;        // the concave shape is a triangle mesh (CmDesc), not a height field
// A mesh item's "rectangle" is (0, triangles overlapped, 0, 1); its tests
// take the triangles in the order of the mesh tree's stack query.
// A triangle test's record: 7 float4, slot-major inside each batch: the
// three vertices, the face normal, the three vertex normals.
constexpr uint32_t TRI_REC = 7;
constexpr int MESH_STACK = 64;    // traversal stack of a mesh tree query (error bit 1 on overflow)
constexpr uint32_t HF_MAX_MANIFOLDS = 4;   // NB_MAX_CONTACT_MANIFOLDS (configuration.h:137)
constexpr uint32_t HF_OUT_POINTS = 16;     // 4 manifolds x 4 points per pair

struct HfRectArgs {
    uint32_t n;
    const int4* items;
    const int32_t* c_shape;
    const rp3dg_shape* shapes;
    const float4* bounds;      // 2 per shape (local bounds)
    const float4 *c_wpos, *c_wori;
    const HfDesc* hf;
    const CmDesc* cm;
    int4* rect;                // out: iMin, iMax, jMin, jMax (mesh: 0, count, 0, 1)
    uint32_t* error;           // bit 1: a mesh tree query overflowed its stack
};

// The triangles of the mesh items, in query order, at their first tests.
struct HfListArgs {
    uint32_t n;
    const int4* items;
    const uint32_t* start;
    const int32_t* c_shape;
    const rp3dg_shape* shapes;
    const float4* bounds;
    const float4 *c_wpos, *c_wori;
    const CmDesc* cm;
    int32_t* tri_id;           // out: per test of a mesh item, its triangle index
    uint32_t* error;
};

struct HfTestArgs {
    uint32_t n_items, n_tests;
    const int4* items;
    const int4* rect;
    const uint32_t* start;     // n_items + 1: first test of each item (concave region)
    const int4* batch;         // per item: x = first test of its algorithm batch, y = batch size
    const int32_t* prev_start; // per item: its first test in the previous step's records (-1: none)
    const int4* prev_rect;     // per item: the rectangle of that step
    const int32_t* c_shape;
    const float4 *c_wpos, *c_wori;
    const HfDesc* hf;
    const CmDesc* cm;
    const int32_t* tri_id;       // mesh items: triangle of each test
    const int32_t* prev_tri_id;  // and of the previous step's tests
    uint32_t* error;             // bit 1: a test named no triangle of its mesh
    const rp3dg_lastframe* prev_cache;
    // outputs: test arrays of the concave region
    int32_t *s1, *s2;
    float4 *p1, *r1, *p2, *r2;
    uint8_t* report;
    rp3dg_lastframe* cache;
    float4* tri;               // TRI_REC float4 per test, slot-major inside each batch
};

struct HfManifoldArgs {
    uint32_t n_items;
    const int4* items;
    const uint32_t* start;
    const int4* batch;             // per item: x = first test of its algorithm batch, y = batch size
    const float4* c_wori;
    float cos_similar;
    const uint8_t* is_colliding;   // concave region
    const uint8_t* nb_contacts;
    const float4 *nd, *l1, *l2;    // concave region outputs, slot-major per batch
    rp3dg_lastframe* cache;
    uint8_t* mid;                  // 16 x n_tests scratch
    uint8_t* out_coll;             // per item
    uint8_t* out_nman;
    uchar4* out_npts;
    float4 *out_nd, *out_l1, *out_l2;   // 16 per item
};

cudaError_t launch_hf_rects(const HfRectArgs& a, cudaStream_t s);
cudaError_t launch_hf_list(const HfListArgs& a, cudaStream_t s);
cudaError_t launch_hf_tests(const HfTestArgs& a, cudaStream_t s);
cudaError_t launch_hf_manifolds(const HfManifoldArgs& a, cudaStream_t s);

}  // namespace rp3dg
