// Kernel-launch interface between the host runtime and the narrow-phase kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"
#include "rp3dg_internal.h"

namespace rp3dg {

constexpr int NP_BLOCK = 128;
// Mesh arenas up to this size are staged in shared memory by every CTA.
constexpr uint32_t MESH_STAGE_MAX_BYTES = 96 * 1024;

struct NpArgs {
    uint32_t n;
    uint32_t nb_shapes;
    uint32_t* error;  // device word: bit 0 = a pair named a shape outside the table
    uint32_t max_contacts;
    int clip;
    int stage_mesh;
    uint32_t mesh_nwords;
    const uint32_t* mesh_words;
    const rp3dg_shape* shapes;
    const int32_t* shape1;
    const int32_t* shape2;
    const float4* pos1;
    const float4* rot1;
    const float4* pos2;
    const float4* rot2;
    const uint8_t* report;
    rp3dg_lastframe* cache;
    uint8_t* is_colliding;
    uint8_t* nb_contacts;
    float4* normal_depth;
    float4* local1;
    float4* local2;
    const void* mlp;                 // packed MLP weights (MlpPacked), read by narrowphase_propose
    const uint8_t* proposals;        // per-pair learned proposal (15 = none) or nullptr
    unsigned long long* mlp_stats;   // [0] proposals tested, [1] confirmed
    // triangle tests (launch_narrowphase_tri): the triangle side of a test has
    // shape index -1; 7 float4 per test, slot-major (k * n + i): the three
    // vertices, the face normal and the three vertex normals
    const float4* tri;
    // polyhedron batches: the order in which the tiles take the pairs (thread
    // t of the batch processes pair perm[t]) or nullptr for 0..n-1
    const uint32_t* perm;
    // event-counting build only: NP_EVENT_COUNT counters (NpEvent order) the
    // kernels add each pair's path events to; ignored by the product kernels
    unsigned long long* events = nullptr;
    // polyhedron batches (required): the thread-per-pair launch does the
    // box-box pairs and appends each pair with a convex mesh to the list of
    // its shape combination c (mesh-box 1, box-mesh 2, mesh-mesh 3) at
    // plist[(c - 1) * n + k], counted in work[c - 1]; the persistent
    // warp-per-pair launch of combination c takes them one at a time
    // (counter work[3 + c - 1])
    uint32_t* plist = nullptr;
    uint32_t* work = nullptr;
};

void upload_box_tables(const BoxTables& t, cudaStream_t s);

// A batch's contacts packed densely for the copy to the host: the pairs in
// groups of 32 (group g = pairs 32g .. 32g + 31); group g's contacts are
// records warp_start[g] ... in pair order, slot order inside a pair, each
// record three float4 (normal and depth, local point 1, local point 2).
// *counter (zeroed before) ends as the number of records.
struct CompactArgs {
    uint32_t n;
    const uint8_t* nb;                    // contacts per pair
    const float4 *nd, *l1, *l2;           // slot-major, n pairs per slot
    float4* records;                      // 3 per record
    uint32_t* warp_start;                 // (n + 31) / 32
    uint32_t* counter;
};
cudaError_t launch_compact_contacts(const CompactArgs& a, cudaStream_t s);
// Launches the kernels of one algorithm batch; *launches receives how many.
cudaError_t launch_narrowphase(int algo, const NpArgs& args, int num_sms, cudaStream_t stream, int* launches);
// Pairs of an all-box polyhedron batch grouped by their learned class
// (colliding first, then the proposed features): perm receives the order
// (the identity when a pair holds a convex mesh); counts is scratch for 32
// words.
cudaError_t launch_partition_by_class(const NpArgs& a, const uint8_t* cls, uint32_t* counts, uint32_t* perm,
                                      cudaStream_t stream);
// Order key of every pair of a polyhedron batch (launch_partition_by_class
// then sorts by it) and, with args.mlp set and proposals non-null, the
// learned proposal of every pair (MLP inference on the tensor cores).
cudaError_t launch_classify_pairs(const NpArgs& a, uint8_t* key, uint8_t* proposals, int num_sms, cudaStream_t stream);
// Triangle tests of one algorithm batch (4, 5 or 6), one test per thread.
cudaError_t launch_narrowphase_tri(int algo, const NpArgs& args, int num_sms, cudaStream_t stream);


}  // namespace rp3dg

// The event-counting build of the narrow-phase kernels (narrowphase_events.cu):
// the same launches as rp3dg::launch_narrowphase / launch_narrowphase_tri /
// upload_box_tables, for an rp3dg::NpArgs whose `events` is set.
cudaError_t rp3dg_events_launch_narrowphase(int algo, const void* args, int num_sms, cudaStream_t stream, int* launches);
cudaError_t rp3dg_events_launch_narrowphase_tri(int algo, const void* args, int num_sms, cudaStream_t stream);
void rp3dg_events_upload_box_tables(const void* t, cudaStream_t stream);
