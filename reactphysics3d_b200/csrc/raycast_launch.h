// Launch interface of the batched world raycast (raycast.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"
#include "rp3dg_internal.h"

namespace rp3dg {

// The world's dynamic AABB tree as RayNode records (rp3dg_internal.h): a
// leaf has child 0 = -2 - collider index.
// Per collider (creation order): x device row of its world transform,
// y body index, z shape index, w collision category bits.
struct RayArgs {
    const RayNode* nodes;
    int32_t root;
    const int4* colliders;
    const float4* c_wpos;          // collider local-to-world position, by row
    const float4* c_wori;          // and orientation
    const rp3dg_shape* shapes;
    const uint32_t* mesh_words;    // convex mesh arena
    const HfDesc* hfields;         // height fields of the context, by id
    uint32_t nb_hfields;
    const CmDesc* cmeshes;         // concave mesh instances of the context, by id
    uint32_t nb_cmeshes;
    const rp3dg_ray* rays;
    uint32_t n;
    int32_t mode;                  // RP3DG_RAYCAST_*
    uint32_t max_hits;
    rp3dg_raycast_hit* hits;       // n * max_hits
    uint32_t* nb_hits;             // n
    uint32_t* error;               // bit 0: a traversal stack overflowed (world or mesh tree)
};

cudaError_t launch_world_raycast(const RayArgs& a, cudaStream_t stream);

}  // namespace rp3dg
