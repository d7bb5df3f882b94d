// Broad phase of a world step: collider world AABBs and the fat-AABB update
// (reference src/systems/BroadPhaseSystem.cpp:155-185,
// src/collision/shapes/CollisionShape.cpp:54-90, SphereShape.cpp:49-58,
// src/collision/broadphase/DynamicAABBTree.cpp:186-214), and the set of
// overlapping pairs of fat AABBs with the pair filters of
// CollisionDetectionSystem::updateOverlappingPairs (:270-343).
//
// The reference keeps the fat AABBs in an incrementally balanced tree and
// queries it for the colliders that moved; the pairs it holds after each step
// are exactly the pairs of overlapping fat AABBs that pass the filters (a
// pair is created or dropped only when one of its colliders is reinserted,
// which is when its fat AABB changes).  Here that set is computed directly:
// an LSD radix sort of the colliders by (group, fat min on the sweep axis),
// then a sweep where each collider scans forward while the next minimum is
// within its maximum, a count pass, an exclusive scan and a write pass, so
// the output order is deterministic.
#include <cuda_runtime.h>

#include "broadphase_launch.h"
#include "rp3dg_math.cuh"
#include "shape_aabb.cuh"

namespace rp3dg {

namespace {

// ---- world AABB + fat AABB update, one collider per thread --------------
__global__ void __launch_bounds__(128) bp_update_kernel(const BpArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_update) return;
    if (a.enabled && !a.enabled[i]) {
        a.moved[i] = 0;
        return;
    }
    const int32_t si = a.shape[i];
    if (uint32_t(si) >= a.nb_shapes) {
        atomicOr(a.error, 1u);
        a.moved[i] = 0;
        return;
    }
    const rp3dg_shape s = a.shapes[si];
    const float4 p4 = a.wpos[i], q4 = a.wori[i];
    v3 amin, amax;
    shape_transformed_aabb(s.kind, s.params[0], a.bounds[2 * si], a.bounds[2 * si + 1],
                           X(V(p4.x, p4.y, p4.z), Q(q4.x, q4.y, q4.z, q4.w)), amin, amax);
    // DynamicAABBTree::updateObject: keep the fat AABB while it contains the
    // new one (AABB::contains), else inflate the new one by 4% of its extent
    // on each side (DYNAMIC_TREE_FAT_AABB_INFLATE_PERCENTAGE 0.08 x 0.5)
    const float4 fmn = a.fat_min[i], fmx = a.fat_max[i];
    const bool inside = fmn.x <= amin.x && fmn.y <= amin.y && fmn.z <= amin.z && fmx.x >= amax.x &&
                        fmx.y >= amax.y && fmx.z >= amax.z;
    const bool force = a.force && a.force[i];
    if (!force && inside) {
        a.moved[i] = 0;
        return;
    }
    const v3 ext = V(amax.x - amin.x, amax.y - amin.y, amax.z - amin.z);
    const v3 gap = V(0.5f * (0.08f * ext.x), 0.5f * (0.08f * ext.y), 0.5f * (0.08f * ext.z));
    a.fat_min[i] = make_float4(amin.x - gap.x, amin.y - gap.y, amin.z - gap.z, 0.0f);
    a.fat_max[i] = make_float4(amax.x + gap.x, amax.y + gap.y, amax.z + gap.z, 0.0f);
    a.moved[i] = 1;
}

// ---- radix sort of 64-bit keys with 32-bit values (LSD, 8-bit digits) ---
constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr uint32_t SORT_TILE = SORT_THREADS * SORT_ITEMS;   // 2048 keys per block
constexpr int SORT_WARPS = SORT_THREADS / 32;

RD uint32_t digit_of(unsigned long long k, int shift) { return uint32_t(k >> shift) & 0xffu; }

__global__ void __launch_bounds__(SORT_THREADS) sort_hist(const unsigned long long* __restrict__ keys, uint32_t n,
                                                          int shift, uint32_t nblocks, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * SORT_TILE;
    for (int k = 0; k < SORT_ITEMS; k++) {
        const uint32_t idx = base + k * SORT_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&h[digit_of(keys[idx], shift)], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of n uint32 in place, one block of 1024 threads (each
// thread scans a contiguous segment).
__global__ void __launch_bounds__(1024) scan_small(uint32_t* __restrict__ v, uint32_t n, uint32_t* __restrict__ total) {
    __shared__ uint32_t part[1024];
    const uint32_t per = (n + 1023) / 1024;
    const uint32_t b = threadIdx.x * per, e = b + per < n ? b + per : n;
    uint32_t s = 0;
    for (uint32_t i = b; i < e; i++) s += v[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        const uint32_t x = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += x;
        __syncthreads();
    }
    uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    for (uint32_t i = b; i < e; i++) {
        const uint32_t x = v[i];
        v[i] = run;
        run += x;
    }
    if (total && threadIdx.x == 1023) *total = part[1023];
}

// Stable scatter: each warp ranks its 256 consecutive keys of the tile in
// order (lanes with equal digits via __match_any_sync), warps are ordered by
// the per-digit counts of the warps before them.
__global__ void __launch_bounds__(SORT_THREADS) sort_scatter(const unsigned long long* __restrict__ keys_in,
                                                             const uint32_t* __restrict__ vals_in,
                                                             unsigned long long* __restrict__ keys_out,
                                                             uint32_t* __restrict__ vals_out, uint32_t n, int shift,
                                                             uint32_t nblocks, const uint32_t* __restrict__ offs) {
    __shared__ uint32_t cnt[SORT_WARPS][256];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint32_t d = lane; d < 256; d += 32) cnt[warp][d] = 0;
    __syncwarp();
    const uint32_t base = blockIdx.x * SORT_TILE + warp * (SORT_ITEMS * 32);
    unsigned long long k_[SORT_ITEMS];
    uint32_t v_[SORT_ITEMS], rank[SORT_ITEMS], dg[SORT_ITEMS];
    const uint32_t lt = (1u << lane) - 1u;
    for (int r = 0; r < SORT_ITEMS; r++) {
        const uint32_t idx = base + r * 32 + lane;
        const bool valid = idx < n;
        k_[r] = valid ? keys_in[idx] : 0ull;
        v_[r] = valid ? vals_in[idx] : 0u;
        const uint32_t d = valid ? digit_of(k_[r], shift) : 256u;
        dg[r] = d;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = valid ? cnt[warp][d] : 0u;
        rank[r] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && (peers & lt) == 0) cnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: counts of the earlier warps of this block
    __shared__ uint32_t woff[SORT_WARPS][256];
    {
        const uint32_t d = threadIdx.x;  // 256 threads, one digit each
        uint32_t run = 0;
        for (int w = 0; w < SORT_WARPS; w++) {
            woff[w][d] = run;
            run += cnt[w][d];
        }
    }
    __syncthreads();
    for (int r = 0; r < SORT_ITEMS; r++) {
        const uint32_t d = dg[r];
        if (d < 256u) {
            const uint32_t pos = offs[d * nblocks + blockIdx.x] + woff[warp][d] + rank[r];
            keys_out[pos] = k_[r];
            vals_out[pos] = v_[r];
        }
    }
}

// ---- sweep ---------------------------------------------------------------

// float -> unsigned key with the same order (negative floats reversed)
RD uint32_t ordered_bits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(128) sap_keys(const BpArgs a, int axis) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float4 mn = a.fat_min[i];
    const float x = axis == 0 ? mn.x : (axis == 1 ? mn.y : mn.z);
    uint32_t g = a.group ? uint32_t(a.group[i]) : 0u;
    if (a.group_bits < 32 && (g >> a.group_bits) != 0u) {
        atomicOr(a.error, 8u);  // group outside 0..nb_groups-1: its pairs are not searched correctly
        g &= (1u << a.group_bits) - 1u;
    }
    a.keys[i] = (static_cast<unsigned long long>(g) << 32) | ordered_bits(x);
    a.vals[i] = i;
}

// Sorted copies of what the sweep reads, sweep axis first.
__global__ void __launch_bounds__(128) sap_gather(const BpArgs a, int axis) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const uint32_t i = a.vals[p];
    const float4 mn = a.fat_min[i], mx = a.fat_max[i];
    float4 lo = mn, hi = mx;
    if (axis == 1) { lo = make_float4(mn.y, mn.x, mn.z, 0.0f); hi = make_float4(mx.y, mx.x, mx.z, 0.0f); }
    if (axis == 2) { lo = make_float4(mn.z, mn.y, mn.x, 0.0f); hi = make_float4(mx.z, mx.y, mx.x, 0.0f); }
    lo.w = __int_as_float(a.body[i]);
    const uint32_t cat = a.category ? a.category[i] : 0xffffu;
    const uint32_t msk = a.mask ? a.mask[i] : 0xffffu;
    hi.w = __uint_as_float((cat << 16) | msk);
    a.s_lo[p] = lo;
    a.s_hi[p] = hi;
    a.s_group[p] = a.group ? a.group[i] : 0;
}

template <bool WRITE>
__global__ void __launch_bounds__(128) sap_sweep(const BpArgs a) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const float4 lo = a.s_lo[p], hi = a.s_hi[p];
    const int32_t g = a.s_group[p];
    const int32_t body = __float_as_int(lo.w);
    const uint32_t bits = __float_as_uint(hi.w);
    const uint32_t cat = bits >> 16, msk = bits & 0xffffu;
    uint32_t count = 0;
    uint32_t out = WRITE ? a.pair_offset[p] : 0u;
    const uint32_t ci = WRITE ? a.vals[p] : 0u;
    for (uint32_t q = p + 1; q < a.n; q++) {
        const float4 lo2 = a.s_lo[q];
        if (lo2.x > hi.x || a.s_group[q] != g) break;   // sorted by (group, min): nothing further overlaps
        const float4 hi2 = a.s_hi[q];
        // AABB::testCollision (AABB.h:179-187) on the two other axes
        if (hi.y < lo2.y || hi2.y < lo.y) continue;
        if (hi.z < lo2.z || hi2.z < lo.z) continue;
        if (__float_as_int(lo2.w) == body) continue;            // same body
        const uint32_t bits2 = __float_as_uint(hi2.w);
        if ((msk & (bits2 >> 16)) == 0u || (cat & (bits2 & 0xffffu)) == 0u) continue;
        if (WRITE) {
            if (out < a.capacity) {
                const uint32_t cj = a.vals[q];
                a.pairs[2 * out] = int32_t(ci < cj ? ci : cj);
                a.pairs[2 * out + 1] = int32_t(ci < cj ? cj : ci);
            }
            out++;
        } else {
            count++;
        }
    }
    if (!WRITE) a.pair_offset[p] = count;
}

uint32_t blocks128(uint32_t n) { return (n + 127) / 128; }

}  // namespace

cudaError_t launch_bp_update(const BpArgs& a, cudaStream_t s, uint64_t* launches) {
    if (a.n_update == 0) return cudaSuccess;
    bp_update_kernel<<<blocks128(a.n_update), 128, 0, s>>>(a);
    (*launches)++;
    return cudaGetLastError();
}

size_t sort_scratch_words(uint32_t n) { return size_t(256) * ((n + SORT_TILE - 1) / SORT_TILE) + 1; }

cudaError_t launch_bp_pairs(const BpArgs& a, int axis, cudaStream_t s, uint64_t* launches) {
    if (a.n == 0) return cudaMemsetAsync(a.pair_count, 0, sizeof(uint32_t), s);
    sap_keys<<<blocks128(a.n), 128, 0, s>>>(a, axis);
    (*launches)++;
    // radix sort (group, min): 32 float bits + the group bits in use
    const uint32_t nblocks = (a.n + SORT_TILE - 1) / SORT_TILE;
    unsigned long long *kin = a.keys, *kout = a.keys_tmp;
    uint32_t *vin = a.vals, *vout = a.vals_tmp;
    const int end_bit = 32 + a.group_bits;
    for (int shift = 0; shift < end_bit; shift += 8) {
        sort_hist<<<nblocks, SORT_THREADS, 0, s>>>(kin, a.n, shift, nblocks, a.sort_hist);
        scan_small<<<1, 1024, 0, s>>>(a.sort_hist, 256 * nblocks, nullptr);
        sort_scatter<<<nblocks, SORT_THREADS, 0, s>>>(kin, vin, kout, vout, a.n, shift, nblocks, a.sort_hist);
        *launches += 3;
        unsigned long long* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
    }
    BpArgs b = a;
    b.keys = kin;
    b.vals = vin;
    sap_gather<<<blocks128(a.n), 128, 0, s>>>(b, axis);
    sap_sweep<false><<<blocks128(a.n), 128, 0, s>>>(b);
    scan_small<<<1, 1024, 0, s>>>(b.pair_offset, a.n, a.pair_count);
    sap_sweep<true><<<blocks128(a.n), 128, 0, s>>>(b);
    *launches += 5;
    return cudaGetLastError();
}

}  // namespace rp3dg
