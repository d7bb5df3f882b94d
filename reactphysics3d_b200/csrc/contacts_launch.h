// Launch interface of the contact-manifold kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"

namespace rp3dg {

struct ReduceArgs {
    uint32_t n;
    uint32_t max_contacts;
    const float4* rot1;      // shape-1 orientations of the pairs
    rp3dg_lastframe* cache;  // temporal-coherence records to update, or nullptr
    uint8_t* is_colliding;
    uint8_t* nb_contacts;
    float4* normal_depth;
    float4* local1;
    float4* local2;
    uint8_t* kept;           // n x 4 kept slot indices (255 = none) or nullptr
};

cudaError_t launch_contacts_reduce(const ReduceArgs& a, cudaStream_t s);

}  // namespace rp3dg
