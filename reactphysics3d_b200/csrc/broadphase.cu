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
// which is when its fat AABB changes).  Here that set is computed directly,
// two ways:
//   - LBVH (the default): 30-bit Morton codes of the fat-AABB centres with
//     the group (world) in the bits above, an LSD radix sort, a Karras tree
//     over the sorted keys (ties broken by sorted position), a bottom-up refit
//     with one atomic visit counter per node, and a traversal in which the 32
//     lanes of a warp hold 32 Morton-consecutive colliders and walk one shared
//     stack (a node is opened when any lane's fat AABB overlaps it; a lane
//     only looks for partners later in the sorted order, so each pair is
//     found once), with a count pass, an exclusive scan and a write pass;
//   - sort and sweep along one axis: an LSD radix sort of the colliders by
//     (group, fat min on the sweep axis), then each collider scans forward
//     while the next minimum is within its maximum.
// Both give the output in a deterministic order.
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

// ---- LBVH -----------------------------------------------------------------

RD float3 aabb_centre(const float4 mn, const float4 mx) {
    return make_float3(0.5f * (mn.x + mx.x), 0.5f * (mn.y + mx.y), 0.5f * (mn.z + mx.z));
}

// Scene bounds of the centres (ordered-bit atomics: min in [0..2], max in [3..5]).
__global__ void __launch_bounds__(128) lbvh_bounds(const BpArgs a, uint32_t* __restrict__ bounds) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
    if (i < a.n) {
        const float3 c = aabb_centre(a.fat_min[i], a.fat_max[i]);
        lo[0] = hi[0] = ordered_bits(c.x);
        lo[1] = hi[1] = ordered_bits(c.y);
        lo[2] = hi[2] = ordered_bits(c.z);
    }
    for (int k = 0; k < 3; k++) {
        for (int o = 16; o; o >>= 1) {
            lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; k++) {
            atomicMin(bounds + k, lo[k]);
            atomicMax(bounds + 3 + k, hi[k]);
        }
    }
}

RD float from_ordered_bits(uint32_t u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }

// 10 bits per axis spread to every third bit
RD uint32_t spread3(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

RD uint32_t quantize10(float x, float lo, float inv) {
    float q = (x - lo) * inv;
    q = q < 0.0f ? 0.0f : (q > 1023.0f ? 1023.0f : q);   // NaN centres land in cell 0
    return uint32_t(q);
}

__global__ void __launch_bounds__(128) lbvh_keys(const BpArgs a, const uint32_t* __restrict__ bounds) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    float lo[3], inv[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = from_ordered_bits(bounds[k]);
        const float ext = from_ordered_bits(bounds[3 + k]) - lo[k];
        inv[k] = ext > 0.0f ? 1023.0f / ext : 0.0f;
    }
    const float3 c = aabb_centre(a.fat_min[i], a.fat_max[i]);
    const uint32_t m = (spread3(quantize10(c.x, lo[0], inv[0])) << 2) | (spread3(quantize10(c.y, lo[1], inv[1])) << 1) |
                       spread3(quantize10(c.z, lo[2], inv[2]));
    uint32_t g = a.group ? uint32_t(a.group[i]) : 0u;
    if (a.group_bits < 32 && (g >> a.group_bits) != 0u) {
        atomicOr(a.error, 8u);  // group outside 0..nb_groups-1
        g &= (1u << a.group_bits) - 1u;
    }
    a.keys[i] = (static_cast<unsigned long long>(g) << 30) | m;
    a.vals[i] = i;
}

// Common-prefix length of sorted keys i and j (Karras 2012), with the sorted
// position breaking ties; -1 outside [0, n).
RD int lbvh_delta(const unsigned long long* __restrict__ k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const unsigned long long ki = k[i], kj = k[j];
    if (ki == kj) return 64 + __clz(uint32_t(i) ^ uint32_t(j));
    return __clzll(ki ^ kj);
}

// Internal node i of the n - 1: its sorted range and its two children
// (internal index, or n - 1 + sorted position for a leaf); node 0 is the root.
__global__ void __launch_bounds__(128) lbvh_build(const unsigned long long* __restrict__ keys, uint32_t n,
                                                  int2* __restrict__ child, int2* __restrict__ range,
                                                  int32_t* __restrict__ parent) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t N = n;
    if (i >= N - 1) return;
    const int d = (lbvh_delta(keys, N, i, i + 1) - lbvh_delta(keys, N, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = lbvh_delta(keys, N, i, i - d);
    int64_t lmax = 2;
    while (lbvh_delta(keys, N, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
        if (lbvh_delta(keys, N, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = lbvh_delta(keys, N, i, j);
    int64_t s = 0, t = l;
    for (;;) {
        t = (t + 1) >> 1;
        if (lbvh_delta(keys, N, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int64_t gamma = i + s * d + (d < 0 ? -1 : 0);
    const int64_t first = i < j ? i : j, last = i < j ? j : i;
    const int32_t left = int32_t(first == gamma ? (N - 1) + gamma : gamma);
    const int32_t right = int32_t(last == gamma + 1 ? (N - 1) + gamma + 1 : gamma + 1);
    child[i] = make_int2(left, right);
    range[i] = make_int2(int32_t(first), int32_t(last));
    parent[left] = int32_t(i);
    parent[right] = int32_t(i);
    if (i == 0) parent[0] = -1;
}

// Bottom-up refit: a leaf's thread walks up; at each node the first arriving
// child stops and the second computes the node's box (its sibling's box is
// visible: written before the fence that precedes the counter increment).
__global__ void __launch_bounds__(128) lbvh_refit(const float4* __restrict__ s_lo, const float4* __restrict__ s_hi,
                                                  uint32_t n, const int2* __restrict__ child,
                                                  const int32_t* __restrict__ parent, uint32_t* __restrict__ visits,
                                                  float4* __restrict__ nlo, float4* __restrict__ nhi) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || n < 2) return;
    const int32_t nl = int32_t(n) - 1;
    int32_t x = parent[nl + int32_t(p)];
    while (x >= 0) {
        __threadfence();
        if (atomicAdd(visits + x, 1u) == 0u) return;
        const int2 c = child[x];
        float4 lo0, hi0, lo1, hi1;
        if (c.x >= nl) { lo0 = s_lo[c.x - nl]; hi0 = s_hi[c.x - nl]; }
        else { lo0 = __ldcg(nlo + c.x); hi0 = __ldcg(nhi + c.x); }
        if (c.y >= nl) { lo1 = s_lo[c.y - nl]; hi1 = s_hi[c.y - nl]; }
        else { lo1 = __ldcg(nlo + c.y); hi1 = __ldcg(nhi + c.y); }
        __stcg(nlo + x, make_float4(fminf(lo0.x, lo1.x), fminf(lo0.y, lo1.y), fminf(lo0.z, lo1.z), 0.0f));
        __stcg(nhi + x, make_float4(fmaxf(hi0.x, hi1.x), fmaxf(hi0.y, hi1.y), fmaxf(hi0.z, hi1.z), 0.0f));
        x = parent[x];
    }
}

constexpr int LBVH_STACK = 128;   // > the deepest tree 96-bit keys can give

// AABB::testCollision (AABB.h:179-187): inclusive on every axis
RD bool aabb_overlap(const float4 alo, const float4 ahi, const float4 blo, const float4 bhi) {
    if (ahi.x < blo.x || bhi.x < alo.x) return false;
    if (ahi.y < blo.y || bhi.y < alo.y) return false;
    if (ahi.z < blo.z || bhi.z < alo.z) return false;
    return true;
}

template <bool WRITE>
__global__ void __launch_bounds__(128) lbvh_query(const BpArgs a, const int2* __restrict__ child,
                                                  const int2* __restrict__ range, const float4* __restrict__ nlo,
                                                  const float4* __restrict__ nhi) {
    __shared__ int32_t stack[4][LBVH_STACK];
    const uint32_t n = a.n;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x * blockDim.x + warp * 32u >= n) return;   // whole warp past the end
    const bool active = p < n;
    const int32_t nl = int32_t(n) - 1;
    float4 qlo = make_float4(0.0f, 0.0f, 0.0f, 0.0f), qhi = qlo;
    int32_t g = 0;
    if (active) { qlo = a.s_lo[p]; qhi = a.s_hi[p]; g = a.s_group[p]; }
    const int32_t body = __float_as_int(qlo.w);
    const uint32_t bits = __float_as_uint(qhi.w);
    const uint32_t cat = bits >> 16, msk = bits & 0xffffu;
    uint32_t count = 0;
    uint32_t out = (WRITE && active) ? a.pair_offset[p] : 0u;
    const uint32_t ci = active ? a.vals[p] : 0u;
    int32_t* st = stack[warp];
    int sp = 0;
    if (n >= 2) { if (lane == 0) st[0] = 0; sp = 1; }
    __syncwarp();
    while (sp > 0) {
        const int32_t node = st[--sp];
        __syncwarp();
        if (node >= nl) {
            // a leaf: sorted position j
            const int32_t j = node - nl;
            bool hit = active && j > int32_t(p);
            if (hit) {
                const float4 lo2 = a.s_lo[j], hi2 = a.s_hi[j];
                const uint32_t bits2 = __float_as_uint(hi2.w);
                hit = a.s_group[j] == g && aabb_overlap(qlo, qhi, lo2, hi2) && __float_as_int(lo2.w) != body &&
                      (msk & (bits2 >> 16)) != 0u && (cat & (bits2 & 0xffffu)) != 0u;
            }
            if (hit) {
                if (WRITE) {
                    if (out < a.capacity) {
                        const uint32_t cj = a.vals[j];
                        a.pairs[2 * out] = int32_t(ci < cj ? ci : cj);
                        a.pairs[2 * out + 1] = int32_t(ci < cj ? cj : ci);
                    }
                    out++;
                } else {
                    count++;
                }
            }
            continue;
        }
        const int2 r = range[node];
        bool hit = active && r.y > int32_t(p);
        if (hit) {
            // the node's sorted range holds groups s_group[r.x] .. s_group[r.y]
            hit = g >= a.s_group[r.x] && g <= a.s_group[r.y] && aabb_overlap(qlo, qhi, nlo[node], nhi[node]);
        }
        if (__any_sync(0xffffffffu, hit)) {
            if (sp + 2 > LBVH_STACK) {
                if (lane == 0) atomicOr(a.error, 16u);   // cannot happen for trees of 96-bit keys
                break;
            }
            const int2 c = child[node];
            if (lane == 0) { st[sp] = c.y; st[sp + 1] = c.x; }
            sp += 2;
            __syncwarp();
        }
    }
    if (!WRITE && active) a.pair_offset[p] = count;
}

}  // namespace

cudaError_t launch_bp_update(const BpArgs& a, cudaStream_t s, uint64_t* launches) {
    if (a.n_update == 0) return cudaSuccess;
    bp_update_kernel<<<blocks128(a.n_update), 128, 0, s>>>(a);
    (*launches)++;
    return cudaGetLastError();
}

size_t sort_scratch_words(uint32_t n) { return size_t(256) * ((n + SORT_TILE - 1) / SORT_TILE) + 1; }

cudaError_t launch_exclusive_scan(uint32_t* v, uint32_t n, uint32_t* total, cudaStream_t s) {
    if (n == 0) return total ? cudaMemsetAsync(total, 0, sizeof(uint32_t), s) : cudaSuccess;
    scan_small<<<1, 1024, 0, s>>>(v, n, total);
    return cudaGetLastError();
}

cudaError_t launch_bp_pairs(const BpArgs& a, int axis, cudaStream_t s, uint64_t* launches) {
    if (a.n == 0) return cudaMemsetAsync(a.pair_count, 0, sizeof(uint32_t), s);
    const bool lbvh = axis < 0;
    if (lbvh) {
        cudaError_t e = cudaMemsetAsync(a.lbvh_bounds, 0xff, 3 * sizeof(uint32_t), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(a.lbvh_bounds + 3, 0, 3 * sizeof(uint32_t), s);
        if (e == cudaSuccess && a.n > 1) e = cudaMemsetAsync(a.lbvh_visits, 0, size_t(a.n) * sizeof(uint32_t), s);
        if (e != cudaSuccess) return e;
        lbvh_bounds<<<blocks128(a.n), 128, 0, s>>>(a, a.lbvh_bounds);
        lbvh_keys<<<blocks128(a.n), 128, 0, s>>>(a, a.lbvh_bounds);
        *launches += 2;
    } else {
        sap_keys<<<blocks128(a.n), 128, 0, s>>>(a, axis);
        (*launches)++;
    }
    // radix sort: (group, Morton code) = 30 + group bits, or (group, min) =
    // 32 float bits + the group bits in use
    const uint32_t nblocks = (a.n + SORT_TILE - 1) / SORT_TILE;
    unsigned long long *kin = a.keys, *kout = a.keys_tmp;
    uint32_t *vin = a.vals, *vout = a.vals_tmp;
    const int end_bit = (lbvh ? 30 : 32) + a.group_bits;
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
    sap_gather<<<blocks128(a.n), 128, 0, s>>>(b, lbvh ? 0 : axis);
    *launches += 1;
    if (lbvh) {
        if (a.n > 1) {
            lbvh_build<<<blocks128(a.n - 1), 128, 0, s>>>(kin, a.n, a.lbvh_child, a.lbvh_range, a.lbvh_parent);
            lbvh_refit<<<blocks128(a.n), 128, 0, s>>>(b.s_lo, b.s_hi, a.n, a.lbvh_child, a.lbvh_parent, a.lbvh_visits,
                                                      a.lbvh_nlo, a.lbvh_nhi);
            *launches += 2;
        }
        lbvh_query<false><<<blocks128(a.n), 128, 0, s>>>(b, a.lbvh_child, a.lbvh_range, a.lbvh_nlo, a.lbvh_nhi);
        scan_small<<<1, 1024, 0, s>>>(b.pair_offset, a.n, a.pair_count);
        lbvh_query<true><<<blocks128(a.n), 128, 0, s>>>(b, a.lbvh_child, a.lbvh_range, a.lbvh_nlo, a.lbvh_nhi);
        *launches += 3;
        return cudaGetLastError();
    }
    sap_sweep<false><<<blocks128(a.n), 128, 0, s>>>(b);
    scan_small<<<1, 1024, 0, s>>>(b.pair_offset, a.n, a.pair_count);
    sap_sweep<true><<<blocks128(a.n), 128, 0, s>>>(b);
    *launches += 3;
    return cudaGetLastError();
}

}  // namespace rp3dg
