// Launch interface of the broad-phase kernels (broadphase.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"

namespace rp3dg {

struct BpArgs {
    uint32_t n;           // colliders in the broad phase
    uint32_t n_update;    // colliders [0, n_update) get new AABBs
    const uint8_t* enabled;  // or null; else only the flagged rows of [0, n_update)
    uint32_t nb_shapes;
    const rp3dg_shape* shapes;
    const float4* bounds;   // 2 per shape: local bounds min, max (CollisionShape::getLocalBounds)
    const int32_t* shape;
    const float4 *wpos, *wori;
    const uint8_t* force;
    float4 *fat_min, *fat_max;
    uint8_t* moved;
    uint32_t* error;
    // pair search
    const int32_t* group;
    const int32_t* body;
    const uint16_t *category, *mask;
    int group_bits;
    unsigned long long *keys, *keys_tmp;
    uint32_t *vals, *vals_tmp;
    uint32_t* sort_hist;
    float4 *s_lo, *s_hi;
    int32_t* s_group;
    uint32_t* pair_offset;
    int32_t* pairs;
    uint32_t capacity;
    uint32_t* pair_count;
    // LBVH (sweep axis < 0): centre bounds (6 words), per internal node its
    // children, sorted range, box and visit counter, per node its parent
    uint32_t* lbvh_bounds;
    int2* lbvh_child;
    int2* lbvh_range;
    int32_t* lbvh_parent;     // 2n - 1 entries
    uint32_t* lbvh_visits;
    float4 *lbvh_nlo, *lbvh_nhi;
};

cudaError_t launch_bp_update(const BpArgs& a, cudaStream_t s, uint64_t* launches);
// axis 0, 1, 2: sort and sweep along that axis; axis < 0: LBVH
cudaError_t launch_bp_pairs(const BpArgs& a, int axis, cudaStream_t s, uint64_t* launches);
// uint32 words of sort histogram scratch for n keys
size_t sort_scratch_words(uint32_t n);
// Exclusive scan of n words in place (one CTA); *total (device, or null) gets the sum.
cudaError_t launch_exclusive_scan(uint32_t* v, uint32_t n, uint32_t* total, cudaStream_t s);

}  // namespace rp3dg
