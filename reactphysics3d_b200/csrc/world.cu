// World step: PhysicsWorld::update (reference src/engine/PhysicsWorld.cpp:
// 239-307) for worlds of convex colliders without joints.
//
// Split of the work.  Everything that is floating-point arithmetic on bodies,
// colliders or contacts runs on the GPU, through the context's device entry
// points (rp3dg_narrowphase_device, rp3dg_reduce_contacts_device,
// rp3dg_dynamics_step_device, rp3dg_broadphase_update_device) and the kernels
// of this file (gathering the narrow-phase batches from the collider arrays,
// packing contact manifolds and points in island order with the warm start of
// initContactsWithPreviousOnes, permuting component rows).  The host keeps the
// structures whose history decides the order of that work (world_order.h: the
// broad-phase tree, the moved-collider set, component order) and the
// reference's bookkeeping around them:
//   computeBroadPhase / updateOverlappingPairs / removeNonOverlappingPairs
//     (CollisionDetectionSystem.cpp:103-343) with the persistent pair arrays of
//     OverlappingPairs (OverlappingPairs.cpp:170-300, 397-449),
//   computeMiddlePhase for convex pairs (:346-410),
//   processPotentialContacts' contact-pair creation (:1198-1260) and
//     addContactPairsToBodies (:714-724),
//   PhysicsWorld::createIslands (PhysicsWorld.cpp:695-866),
//   createContacts' packing order (CollisionDetectionSystem.cpp:906-975),
//   BroadPhaseSystem::updateColliders' reinsertions (BroadPhaseSystem.cpp:
//     130-185),
//   PhysicsWorld::updateSleepingBodies (PhysicsWorld.cpp:871-926) with
//     RigidBody::setIsSleeping (RigidBody.cpp:1006-1057) and the pair
//     enable/disable of RigidBody.cpp:1060-1140.
// Two synchronisations per step bring back what that bookkeeping reads: the
// narrow-phase outcome (colliding flag and kept point count per tested pair)
// and, after the step, the broad-phase reinsertion flags, the new fat AABBs
// and the velocities (sleep test).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/rp3dg.h"
#include "rp3dg_math.cuh"
#include "world_order.h"

namespace rp3dg {
// host copy of the context's shape table (rp3dg_host.cu)
int get_shapes_host(rp3dg_ctx* ctx, std::vector<rp3dg_shape>* out);
void set_error(rp3dg_ctx* ctx, const std::string& msg);
}  // namespace rp3dg

using rp3dg::order::Box;
using namespace rp3dg;

namespace {

constexpr int NB_ALGOS = 6;
constexpr uint32_t MAXC = RP3DG_MAX_CONTACTS_PER_PAIR;

// ---------------------------------------------------------------- kernels

struct GatherArgs {
    uint32_t n;
    const int4* items;          // x collider-1 row, y collider-2 row, z cache slot, w report flag
    const int32_t* c_shape;
    const float4 *c_wpos, *c_wori;
    const rp3dg_lastframe* pool;
    int32_t *s1, *s2;
    float4 *p1, *r1, *p2, *r2;
    uint8_t* report;
    rp3dg_lastframe* cache;
};

// Narrow-phase batch of the middle phase: shapes and local-to-world
// transforms of the two colliders and the pair's temporal-coherence record.
__global__ void __launch_bounds__(128) world_gather_batch(const GatherArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int4 it = a.items[i];
    a.s1[i] = a.c_shape[it.x];
    a.s2[i] = a.c_shape[it.y];
    a.p1[i] = a.c_wpos[it.x];
    a.r1[i] = a.c_wori[it.x];
    a.p2[i] = a.c_wpos[it.y];
    a.r2[i] = a.c_wori[it.y];
    a.report[i] = uint8_t(it.w);
    a.cache[i] = a.pool[it.z];
}

__global__ void __launch_bounds__(128) world_scatter_cache(uint32_t n, const int4* items, const rp3dg_lastframe* cache,
                                                           rp3dg_lastframe* pool) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pool[items[i].z] = cache[i];
}

// LastFrameCollisionInfo() of a new overlapping pair (OverlappingPairs.h:86-91).
__global__ void __launch_bounds__(128) world_reset_cache(uint32_t n, const int32_t* slots, rp3dg_lastframe* pool) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rp3dg_lastframe f;
    f.gjk_axis[0] = 0.0f;
    f.gjk_axis[1] = 1.0f;
    f.gjk_axis[2] = 0.0f;
    f.flags = 0;
    f.sat_face = 0;
    f.sat_edge1 = 0;
    f.sat_edge2 = 0;
    pool[slots[i]] = f;
}

struct PackArgs {
    uint32_t nm;
    const int4* ids;            // body1 row, body2 row, collider1 row, collider2 row
    const int4* src;            // x item index inside its batch, y batch size, z batch first item, w first point
    const int4* prev;           // previous pair's manifold start, count, point start, count (x < 0: none)
    const uint8_t* kept_count;  // points kept by the manifold step, per item
    const float4 *b_nd, *b_l1, *b_l2;  // narrow-phase outputs, slot-major per batch (16 slots)
    float cos_similar, persist2;
    // previous step's manifolds and points (after storeImpulses)
    const uint32_t* pm_pstart;
    const float4 *pm_fv1, *pm_fv2, *pm_fimp;
    const float4 *pp_nd, *pp_l1;
    const float* pp_imp;
    const uint8_t* pp_rest;
    // current arrays
    int4* m_ids;
    uint32_t* m_pstart;
    uint8_t* m_npts;
    float4 *m_fv1, *m_fv2, *m_fimp;
    float4 *p_nd, *p_l1, *p_l2;
    float* p_imp;
    uint8_t* p_rest;
};

// createContacts (CollisionDetectionSystem.cpp:906-960) + the warm start of
// initContactsWithPreviousOnes (:1069-1160) for convex pairs: one manifold
// per contact pair, one thread per manifold.
__global__ void __launch_bounds__(128) world_pack_contacts(const PackArgs a) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.nm) return;
    const int4 s = a.src[m];
    const uint32_t item = uint32_t(s.z + s.x);
    const uint32_t k = a.kept_count[item];
    const uint32_t ps = uint32_t(s.w);
    const uint32_t base = uint32_t(s.z) * MAXC;  // batch region start (float4 units)
    a.m_ids[m] = a.ids[m];
    a.m_pstart[m] = ps;
    a.m_npts[m] = uint8_t(k);
    for (uint32_t c = 0; c < k; c++) {
        const uint32_t src = base + c * uint32_t(s.y) + uint32_t(s.x);
        a.p_nd[ps + c] = a.b_nd[src];
        a.p_l1[ps + c] = a.b_l1[src];
        a.p_l2[ps + c] = a.b_l2[src];
    }
    float4 fv1 = make_float4(0.f, 0.f, 0.f, 0.f), fv2 = fv1, fimp = fv1;
    const int4 pv = a.prev[m];
    if (pv.x >= 0 && k > 0) {
        const float4 cn = a.b_nd[base + uint32_t(s.x)];
        for (int p = pv.x; p < pv.x + pv.y; p++) {
            const float4 pn = a.pp_nd[a.pm_pstart[p]];
            // previousNormal.dot(currentNormal) >= cosAngleSimilarContactManifold
            const float d = pn.x * cn.x + pn.y * cn.y + pn.z * cn.z;
            if (d >= a.cos_similar) {
                fv1 = a.pm_fv1[p];
                fv2 = a.pm_fv2[p];
                fimp = a.pm_fimp[p];
                break;
            }
        }
    }
    a.m_fv1[m] = fv1;
    a.m_fv2[m] = fv2;
    a.m_fimp[m] = fimp;
    for (uint32_t c = 0; c < k; c++) {
        float imp = 0.0f;
        uint8_t rest = 0;
        if (pv.x >= 0) {
            const float4 l = a.p_l1[ps + c];
            for (int p = pv.z; p < pv.z + pv.w; p++) {
                const float4 q = a.pp_l1[p];
                const float dx = l.x - q.x, dy = l.y - q.y, dz = l.z - q.z;
                if (dx * dx + dy * dy + dz * dz <= a.persist2) {
                    imp = a.pp_imp[p];
                    rest = a.pp_rest[p];
                    break;
                }
            }
        }
        a.p_imp[ps + c] = imp;
        a.p_rest[ps + c] = rest;
    }
}

// Row permutation after component swaps: dst[r] = src[perm[r]] for each of
// the listed float4 columns (w float4 per row).
struct PermCol {
    const float4* src;
    float4* dst;
    int w;
};
struct PermArgs {
    uint32_t n;
    const int32_t* perm;
    int ncol;
    PermCol col[16];
};
__global__ void __launch_bounds__(128) world_permute(const PermArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.n) return;
    const uint32_t s = uint32_t(a.perm[r]);
    for (int c = 0; c < a.ncol; c++) {
        const int w = a.col[c].w;
        for (int j = 0; j < w; j++) a.col[c].dst[size_t(r) * w + j] = a.col[c].src[size_t(s) * w + j];
    }
}

// Collider local-to-world transforms and body centres of mass at creation
// (Transform * Transform, Transform * Vector3: Transform.h:193-225).
__global__ void __launch_bounds__(128) world_setup(uint32_t nb, const float4* pos, const float4* ori,
                                                   const float4* com_local, float4* com_world, const uint8_t* dynamic,
                                                   uint32_t nc, const int32_t* c_body, const float4* lpos,
                                                   const float4* lori, float4* wpos, float4* wori) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) {
        const float4 p = pos[i], q = ori[i], c = com_local[i];
        if (dynamic[i]) {
            const v3 w = xapply(X(V(p.x, p.y, p.z), Q(q.x, q.y, q.z, q.w)), V(c.x, c.y, c.z));
            com_world[i] = make_float4(w.x, w.y, w.z, 0.0f);
        } else {
            com_world[i] = make_float4(p.x, p.y, p.z, 0.0f);
        }
    }
    if (i < nc) {
        const int32_t b = c_body[i];
        const float4 p = pos[b], q = ori[b], lp = lpos[i], lq = lori[i];
        const xform t = xmul(X(V(p.x, p.y, p.z), Q(q.x, q.y, q.z, q.w)), X(V(lp.x, lp.y, lp.z), Q(lq.x, lq.y, lq.z, lq.w)));
        wpos[i] = make_float4(t.p.x, t.p.y, t.p.z, 0.0f);
        wori[i] = make_float4(t.q.x, t.q.y, t.q.z, t.q.w);
    }
}

// setIsSleeping(true): velocities, forces and torques of the listed rows set
// to zero (RigidBody.cpp:1040-1046).
__global__ void __launch_bounds__(128) world_zero_rows(uint32_t n, const int32_t* rows, float4* lv, float4* av,
                                                       float4* force, float4* torque) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t r = rows[i];
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    lv[r] = z;
    av[r] = z;
    force[r] = z;
    torque[r] = z;
}

uint32_t blocks(uint32_t n) { return (n + 127) / 128; }

// ------------------------------------------------------------------ host

// Volume and local inertia tensor of a shape (BoxShape.h:233, BoxShape.cpp:53-59,
// SphereShape.h:170-178, CapsuleShape.h:175-177, CapsuleShape.cpp:51-67).
bool shape_mass(const rp3dg_shape& s, float mass_density, float* vol_out, float* inertia /*3*/, float* mass_out) {
    const float PI = float(3.141592653589);
    float vol;
    if (s.kind == RP3DG_SHAPE_BOX) {
        vol = 8.0f * s.params[0] * s.params[1] * s.params[2];
    } else if (s.kind == RP3DG_SHAPE_SPHERE) {
        const float r = s.params[0];
        vol = 4.0f / 3.0f * PI * r * r * r;
    } else if (s.kind == RP3DG_SHAPE_CAPSULE) {
        const float r = s.params[0], hh = s.params[1];
        vol = PI * r * r * (4.0f * r / 3.0f + 2.0f * hh);
    } else {
        return false;
    }
    const float mass = vol * mass_density;
    if (s.kind == RP3DG_SHAPE_BOX) {
        const float factor = (1.0f / 3.0f) * mass;
        const float xs = s.params[0] * s.params[0], ys = s.params[1] * s.params[1], zs = s.params[2] * s.params[2];
        inertia[0] = factor * (ys + zs);
        inertia[1] = factor * (xs + zs);
        inertia[2] = factor * (xs + ys);
    } else if (s.kind == RP3DG_SHAPE_SPHERE) {
        const float d = 0.4f * mass * s.params[0] * s.params[0];
        inertia[0] = inertia[1] = inertia[2] = d;
    } else {
        const float r = s.params[0], hh = s.params[1];
        const float height = hh + hh;
        const float r2 = r * r, h2 = height * height, r2d = r2 + r2;
        const float f1 = 2.0f * r / (4.0f * r + 3.0f * height);
        const float f2 = 3.0f * height / (4.0f * r + 3.0f * height);
        const float sum1 = 0.4f * r2d;
        const float sum2 = 0.75f * height * r + 0.5f * h2;
        const float sum3 = 0.25f * r2 + float(1.0 / 12.0) * h2;
        const float ixz = f1 * mass * (sum1 + sum2) + f2 * mass * sum3;
        const float iy = f1 * mass * sum1 + f2 * mass * 0.25f * r2d;
        inertia[0] = ixz;
        inertia[1] = iy;
        inertia[2] = ixz;
    }
    *vol_out = vol;
    *mass_out = mass;
    return true;
}

// Quaternion::getMatrix (Quaternion.cpp:138-165)
void quat_matrix(const float* q, float m[3][3]) {
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    const float nQ = x * x + y * y + z * z + w * w;
    float s = 0.0f;
    if (nQ > 0.0f) s = 2.0f / nQ;
    const float xs = x * s, ys = y * s, zs = z * s;
    const float wxs = w * xs, wys = w * ys, wzs = w * zs;
    const float xxs = x * xs, xys = x * ys, xzs = x * zs;
    const float yys = y * ys, yzs = y * zs, zzs = z * zs;
    m[0][0] = 1.0f - yys - zzs; m[0][1] = xys - wzs;        m[0][2] = xzs + wys;
    m[1][0] = xys + wzs;        m[1][1] = 1.0f - xxs - zzs; m[1][2] = yzs - wxs;
    m[2][0] = xzs - wys;        m[2][1] = yzs + wxs;        m[2][2] = 1.0f - xxs - yys;
}

struct BodyH {
    int type = RP3DG_BODY_DYNAMIC;
    bool sleeping = false;
    bool allowed_sleep = true;
    bool in_island = false;
    bool has_sim_collider = false;
    float sleep_time = 0.0f;
    std::vector<int> colliders;
    std::vector<uint32_t> contact_pairs;
};
struct ColliderH {
    int body = -1;
    int shape = -1;
    int bp = -1;  // broad-phase id (tree leaf)
    uint16_t category = 1, mask = 0xffff;
    std::vector<uint64_t> pairs;  // ColliderComponents::mOverlappingPairs
};
struct PairH {
    uint64_t id = 0;
    int bp1 = -1, bp2 = -1;
    int c1 = -1, c2 = -1;  // collider ids
    int algo = 0;
    bool need_test = false, coll_prev = false, coll_curr = false, enabled = true;
    int cache = -1;  // slot of its LastFrameCollisionInfo in the device pool
};
struct ContactPairH {
    uint64_t id;
    int b1, b2, c1, c2;
    uint32_t item;       // global narrow-phase item
    uint32_t k;          // points after the manifold step
    bool in_island = false;
    uint32_t manifold = 0, point = 0;  // indices in the packed arrays
};
struct IslandH {
    uint32_t manifold_start = 0, manifold_count = 0;
    std::vector<int> bodies;
};

// pairNumbers (mathematics_functions.h:428-433)
inline uint64_t pair_number(uint32_t a, uint32_t b) {
    const uint64_t A = a, B = b;
    return A * A + A + B;
}

template <class T>
int dev_grow(T** p, size_t* cap, size_t need) {
    if (need <= *cap) return 0;
    size_t n = std::max<size_t>(need, *cap * 2);
    n = std::max<size_t>(n, 64);
    cudaFree(*p);
    *p = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)) != cudaSuccess) {
        *cap = 0;
        return -1;
    }
    *cap = n;
    return 0;
}
template <class T>
int host_grow(T** p, size_t* cap, size_t need) {
    if (need <= *cap) return 0;
    size_t n = std::max<size_t>(need, *cap * 2);
    n = std::max<size_t>(n, 64);
    cudaFreeHost(*p);
    *p = nullptr;
    if (cudaMallocHost(reinterpret_cast<void**>(p), n * sizeof(T)) != cudaSuccess) {
        *cap = 0;
        return -1;
    }
    *cap = n;
    return 0;
}

// Device columns of the rigid-body components (row = component slot).
enum BodyCol { BC_POS, BC_ORI, BC_COMW, BC_COML, BC_LV, BC_AV, BC_F, BC_T, BC_IIL, BC_MASS, BC_LLOCK, BC_ALOCK, BC_NCOL };
enum ColCol { CC_LPOS, CC_LORI, CC_WPOS, CC_WORI, CC_MAT, CC_FMIN, CC_FMAX, CC_NCOL };

struct ContactBuf {
    size_t cap_m = 0, cap_p = 0;
    int4* ids = nullptr;
    uint32_t* pstart = nullptr;
    uint8_t* npts = nullptr;
    float4 *fv1 = nullptr, *fv2 = nullptr, *fimp = nullptr;
    float4 *nd = nullptr, *l1 = nullptr, *l2 = nullptr;
    float* imp = nullptr;
    uint8_t* rest = nullptr;
    uint32_t nm = 0, np = 0;
    size_t c_ids = 0, c_ps = 0, c_np = 0, c_fv1 = 0, c_fv2 = 0, c_fimp = 0, c_nd = 0, c_l1 = 0, c_l2 = 0, c_imp = 0,
           c_rest = 0;
    int ensure(uint32_t m, uint32_t p) {
        int rc = 0;
        rc |= dev_grow(&ids, &c_ids, m);
        rc |= dev_grow(&pstart, &c_ps, m);
        rc |= dev_grow(&npts, &c_np, m);
        rc |= dev_grow(&fv1, &c_fv1, m);
        rc |= dev_grow(&fv2, &c_fv2, m);
        rc |= dev_grow(&fimp, &c_fimp, m);
        rc |= dev_grow(&nd, &c_nd, p);
        rc |= dev_grow(&l1, &c_l1, p);
        rc |= dev_grow(&l2, &c_l2, p);
        rc |= dev_grow(&imp, &c_imp, p);
        rc |= dev_grow(&rest, &c_rest, p);
        return rc;
    }
    void release() {
        cudaFree(ids); cudaFree(pstart); cudaFree(npts); cudaFree(fv1); cudaFree(fv2); cudaFree(fimp);
        cudaFree(nd); cudaFree(l1); cudaFree(l2); cudaFree(imp); cudaFree(rest);
    }
};

}  // namespace

struct rp3dg_world {
    rp3dg_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    rp3dg_world_settings set{};
    uint32_t nb = 0, nc = 0;
    std::vector<BodyH> bodies;
    std::vector<ColliderH> colliders;
    std::vector<rp3dg_shape> shapes;
    rp3dg::order::Comps bcomp, ccomp;
    rp3dg::order::Tree tree;
    rp3dg::order::IdSet moved;
    std::vector<int> bp_to_collider;
    // overlapping pairs (OverlappingPairs::mConvexPairs / mDisabledConvexPairs)
    std::vector<PairH> pairs, disabled;
    std::unordered_map<uint64_t, uint32_t> map_pairs, map_disabled;
    std::vector<int> free_cache;
    uint32_t cache_next = 0;
    std::vector<int32_t> reset_slots;
    // contacts of this step and the previous one
    std::vector<ContactPairH> cpairs, prev_cpairs;
    std::unordered_map<uint64_t, uint32_t> prev_map;
    std::vector<uint32_t> island_order;  // mProcessContactPairsOrderIslands
    std::vector<IslandH> islands;
    // device rows currently in the order of these slot lists
    std::vector<int> dev_body_at, dev_col_at;
    // device state
    float4* bcol[2][BC_NCOL] = {};
    float4* biiw[2] = {};
    uint8_t* bgrav = nullptr;
    float4* ccol[2][CC_NCOL] = {};
    int32_t* c_body = nullptr;
    int32_t* c_shape = nullptr;
    uint16_t *c_cat = nullptr, *c_mask = nullptr;
    uint8_t* c_moved = nullptr;
    int cur_b = 0, cur_c = 0;
    rp3dg_lastframe* pool = nullptr;
    size_t cap_pool = 0;
    int32_t* d_small = nullptr;  // reset slots / permutation / rows
    size_t cap_small = 0;
    // narrow-phase step buffers (all batches concatenated)
    size_t cap_items = 0;
    int4* d_items = nullptr;
    int32_t *d_s1 = nullptr, *d_s2 = nullptr;
    float4 *d_p1 = nullptr, *d_r1 = nullptr, *d_p2 = nullptr, *d_r2 = nullptr;
    uint8_t *d_rep = nullptr, *d_coll = nullptr, *d_nct = nullptr;
    rp3dg_lastframe* d_cache = nullptr;
    float4 *d_nd = nullptr, *d_l1 = nullptr, *d_l2 = nullptr;
    // manifold packing inputs
    size_t cap_m = 0;
    int4 *d_mids = nullptr, *d_msrc = nullptr, *d_mprev = nullptr;
    size_t cap_i = 0;
    uint32_t *d_istart = nullptr, *d_icount = nullptr;
    ContactBuf cbuf[2];
    int cur_cb = 0;
    // pinned host staging
    size_t cap_hitems = 0, cap_hm = 0, cap_hi = 0, cap_hstep = 0;
    int4* h_items = nullptr;
    uint8_t* h_out = nullptr;  // colliding flag, kept count
    size_t cap_hout = 0;
    int4 *h_mids = nullptr, *h_msrc = nullptr, *h_mprev = nullptr;
    uint32_t *h_istart = nullptr, *h_icount = nullptr;
    uint8_t* h_step = nullptr;  // moved flags, fat AABBs, velocities after the step
    // batches of this step
    uint32_t batch_start[NB_ALGOS + 1] = {};
    std::vector<int4> items;
    std::vector<uint32_t> item_pair;  // index into pairs of each item
    std::vector<uint8_t> gravity;  // gravity flag by body id (re-uploaded after permutations)
    bool tables_dirty = true;
    // phase profiling (rp3dg_world_set_profiling): cumulative ms per phase
    bool profiling = false;
    double phase_ms[8] = {};
    std::chrono::steady_clock::time_point t_mark;
    rp3dg_world_stats stats{};
    std::string err;
};

namespace {

int wfail(rp3dg_world* w, int code, const std::string& msg) {
    if (w) {
        w->err = msg;
        rp3dg::set_error(w->ctx, "world: " + msg);
    }
    return code;
}
int cfail(rp3dg_ctx* ctx, int code, const std::string& msg) {
    rp3dg::set_error(ctx, "world: " + msg);
    return code;
}
int wcuda(rp3dg_world* w, cudaError_t e, const char* what) {
    return wfail(w, RP3DG_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int shape_type_index(const rp3dg_shape& s) {
    // CollisionShapeType: SPHERE 0, CAPSULE 1, CONVEX_POLYHEDRON 2
    return s.kind == RP3DG_SHAPE_SPHERE ? 0 : s.kind == RP3DG_SHAPE_CAPSULE ? 1 : 2;
}
// CollisionDispatch::selectNarrowPhaseAlgorithm (CollisionDispatch.cpp:80-115, 208-222)
int select_algorithm(int t1, int t2) {
    if (t1 > t2) std::swap(t1, t2);
    if (t1 == 0 && t2 == 0) return RP3DG_ALGO_SPHERE_VS_SPHERE;
    if (t1 == 0 && t2 == 1) return RP3DG_ALGO_SPHERE_VS_CAPSULE;
    if (t1 == 1 && t2 == 1) return RP3DG_ALGO_CAPSULE_VS_CAPSULE;
    if (t1 == 0 && t2 == 2) return RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON;
    if (t1 == 1 && t2 == 2) return RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON;
    return RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON;
}

int alloc_cache(rp3dg_world* w) {
    int slot;
    if (!w->free_cache.empty()) {
        slot = w->free_cache.back();
        w->free_cache.pop_back();
    } else {
        slot = int(w->cache_next++);
    }
    w->reset_slots.push_back(slot);
    return slot;
}

PairH* find_pair(rp3dg_world* w, uint64_t id) {
    auto it = w->map_pairs.find(id);
    if (it != w->map_pairs.end()) return &w->pairs[it->second];
    it = w->map_disabled.find(id);
    if (it != w->map_disabled.end()) return &w->disabled[it->second];
    return nullptr;
}

// swap-remove from a pair array keeping its id map (removeConvexPairWithIndex)
void remove_pair_at(std::vector<PairH>& arr, std::unordered_map<uint64_t, uint32_t>& map, uint32_t idx) {
    map.erase(arr[idx].id);
    const uint32_t last = uint32_t(arr.size()) - 1;
    if (arr.size() > 1 && idx < last) map[arr[last].id] = idx;
    arr[idx] = arr[last];
    arr.pop_back();
}

void remove_from_collider(rp3dg_world* w, int c, uint64_t id) {
    auto& v = w->colliders[size_t(c)].pairs;
    auto it = std::find(v.begin(), v.end(), id);
    if (it != v.end()) v.erase(it);
}

// OverlappingPairs::addPair (OverlappingPairs.cpp:397-449), convex pairs
void add_pair(rp3dg_world* w, int c1, int c2) {
    const uint32_t b1 = uint32_t(w->colliders[size_t(c1)].bp), b2 = uint32_t(w->colliders[size_t(c2)].bp);
    PairH p;
    p.id = pair_number(std::max(b1, b2), std::min(b1, b2));
    p.bp1 = int(b1);
    p.bp2 = int(b2);
    p.c1 = c1;
    p.c2 = c2;
    p.algo = select_algorithm(shape_type_index(w->shapes[size_t(w->colliders[size_t(c1)].shape)]),
                              shape_type_index(w->shapes[size_t(w->colliders[size_t(c2)].shape)]));
    p.enabled = true;
    p.cache = alloc_cache(w);
    w->map_pairs[p.id] = uint32_t(w->pairs.size());
    w->pairs.push_back(p);
    w->colliders[size_t(c1)].pairs.push_back(p.id);
    w->colliders[size_t(c2)].pairs.push_back(p.id);
}

// removeConvexPairWithIndex(index, removeFromColliders = true)
void remove_pair(rp3dg_world* w, uint32_t idx) {
    PairH& p = w->pairs[idx];
    remove_from_collider(w, p.c1, p.id);
    remove_from_collider(w, p.c2, p.id);
    w->free_cache.push_back(p.cache);
    remove_pair_at(w->pairs, w->map_pairs, idx);
}

// disableConvexPairWithIndex / enableConvexPairWithIndex: the pair is
// re-created in the other array with a fresh temporal-coherence record
void disable_pair(rp3dg_world* w, uint64_t id) {
    auto it = w->map_pairs.find(id);
    if (it == w->map_pairs.end()) return;
    const uint32_t idx = it->second;
    PairH np = w->pairs[idx];
    np.enabled = false;
    np.need_test = false;
    w->free_cache.push_back(np.cache);
    np.cache = alloc_cache(w);
    w->map_disabled[id] = uint32_t(w->disabled.size());
    w->disabled.push_back(np);
    remove_pair_at(w->pairs, w->map_pairs, idx);
}
void enable_pair(rp3dg_world* w, uint64_t id) {
    auto it = w->map_disabled.find(id);
    if (it == w->map_disabled.end()) return;
    const uint32_t idx = it->second;
    PairH np = w->disabled[idx];
    np.enabled = true;
    np.need_test = false;
    w->free_cache.push_back(np.cache);
    np.cache = alloc_cache(w);
    w->map_pairs[id] = uint32_t(w->pairs.size());
    w->pairs.push_back(np);
    remove_pair_at(w->disabled, w->map_disabled, idx);
}

// BroadPhaseSystem::addMovedCollider + notifyOverlappingPairsToTestOverlap
void add_moved(rp3dg_world* w, int c) {
    w->moved.add(w->colliders[size_t(c)].bp);
    for (uint64_t id : w->colliders[size_t(c)].pairs) {
        PairH* p = find_pair(w, id);
        if (p) p->need_test = true;
    }
}

// PhysicsWorld::setBodyDisabled (PhysicsWorld.cpp:168-186)
void set_body_disabled(rp3dg_world* w, int b, bool dis) {
    if (w->bcomp.enabled(b) == !dis) return;
    w->bcomp.set_disabled(b, dis);
    for (int c : w->bodies[size_t(b)].colliders) w->ccomp.set_disabled(c, dis);
}

// RigidBody::setIsSleeping (RigidBody.cpp:1006-1057)
void set_sleeping(rp3dg_world* w, int b, bool sleeping, std::vector<int32_t>* zero_rows) {
    BodyH& B = w->bodies[size_t(b)];
    if (B.sleeping == sleeping) return;
    if (B.type == RP3DG_BODY_STATIC) return;
    if (sleeping) B.sleep_time = 0.0f;
    else if (B.sleeping) B.sleep_time = 0.0f;
    B.sleeping = sleeping;
    set_body_disabled(w, b, sleeping);
    if (sleeping) {
        // checkForDisabledOverlappingPairs
        for (int c : B.colliders) {
            const std::vector<uint64_t> ids = w->colliders[size_t(c)].pairs;
            for (uint64_t id : ids) {
                PairH* p = find_pair(w, id);
                if (!p) continue;
                const int o1 = w->colliders[size_t(p->c1)].body, o2 = w->colliders[size_t(p->c2)].body;
                if (!w->bcomp.enabled(o1) && !w->bcomp.enabled(o2)) disable_pair(w, id);
            }
        }
        zero_rows->push_back(b);
    } else {
        // enableOverlappingPairs + askForBroadPhaseCollisionCheck
        for (int c : B.colliders) {
            const std::vector<uint64_t> ids = w->colliders[size_t(c)].pairs;
            for (uint64_t id : ids) {
                PairH* p = find_pair(w, id);
                if (p && !p->enabled) enable_pair(w, id);
            }
        }
        for (int c : B.colliders) add_moved(w, c);
    }
}

// ---------------------------------------------------------------- phases

// computeBroadPhase (CollisionDetectionSystem.cpp:103-167, 270-343)
void broad_phase(rp3dg_world* w) {
    std::vector<int32_t> shapes;
    w->moved.to_array(shapes);
    w->moved.clear();
    std::vector<int> leaves, stack;
    for (int32_t s : shapes) {
        leaves.clear();
        w->tree.query(w->tree.nodes[size_t(s)].box, leaves, stack);
        for (int leaf : leaves) {
            if (leaf == s) continue;
            const int c1 = w->bp_to_collider[size_t(s)], c2 = w->bp_to_collider[size_t(leaf)];
            const ColliderH &C1 = w->colliders[size_t(c1)], &C2 = w->colliders[size_t(c2)];
            if (C1.body == C2.body) continue;
            const uint64_t id = pair_number(uint32_t(std::max(s, leaf)), uint32_t(std::min(s, leaf)));
            PairH* p = find_pair(w, id);
            if (!p) {
                if ((C1.mask & C2.category) != 0 && (C1.category & C2.mask) != 0) add_pair(w, c1, c2);
            } else {
                p->need_test = false;
            }
        }
    }
    // removeNonOverlappingPairs
    for (uint64_t i = 0; i < w->pairs.size(); i++) {
        PairH& p = w->pairs[i];
        if (!p.need_test) continue;
        if (rp3dg::order::overlap(w->tree.nodes[size_t(p.bp1)].box, w->tree.nodes[size_t(p.bp2)].box)) {
            p.need_test = false;
        } else {
            remove_pair(w, uint32_t(i));
            i--;
        }
    }
}

int ensure_items(rp3dg_world* w, size_t n) {
    if (n <= w->cap_items) return 0;
    size_t c = std::max<size_t>(n, w->cap_items * 2);
    c = std::max<size_t>(c, 256);
    cudaFree(w->d_items); cudaFree(w->d_s1); cudaFree(w->d_s2); cudaFree(w->d_p1); cudaFree(w->d_r1);
    cudaFree(w->d_p2); cudaFree(w->d_r2); cudaFree(w->d_rep); cudaFree(w->d_coll); cudaFree(w->d_nct);
    cudaFree(w->d_cache); cudaFree(w->d_nd); cudaFree(w->d_l1); cudaFree(w->d_l2);
    cudaError_t e = cudaSuccess;
    auto M = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, b); };
    M((void**)&w->d_items, c * 16); M((void**)&w->d_s1, c * 4); M((void**)&w->d_s2, c * 4);
    M((void**)&w->d_p1, c * 16); M((void**)&w->d_r1, c * 16); M((void**)&w->d_p2, c * 16); M((void**)&w->d_r2, c * 16);
    M((void**)&w->d_rep, c); M((void**)&w->d_coll, c); M((void**)&w->d_nct, c);
    M((void**)&w->d_cache, c * 16);
    M((void**)&w->d_nd, c * 16 * MAXC); M((void**)&w->d_l1, c * 16 * MAXC); M((void**)&w->d_l2, c * 16 * MAXC);
    if (e != cudaSuccess) { w->cap_items = 0; return wcuda(w, e, "cudaMalloc(narrow-phase step buffers)"); }
    w->cap_items = c;
    if (host_grow(&w->h_items, &w->cap_hitems, c) || host_grow(&w->h_out, &w->cap_hout, 2 * c))
        return wfail(w, RP3DG_ENOMEM, "cudaMallocHost(step staging)");
    return 0;
}

int ensure_pool(rp3dg_world* w) {
    const size_t need = w->cache_next;
    if (need <= w->cap_pool) return 0;
    size_t c = std::max<size_t>(need, w->cap_pool * 2);
    c = std::max<size_t>(c, 1024);
    rp3dg_lastframe* np = nullptr;
    cudaError_t e = cudaMalloc(&np, c * sizeof(rp3dg_lastframe));
    if (e != cudaSuccess) return wcuda(w, e, "cudaMalloc(cache pool)");
    if (w->pool && w->cap_pool)
        cudaMemcpyAsync(np, w->pool, w->cap_pool * sizeof(rp3dg_lastframe), cudaMemcpyDeviceToDevice, w->stream);
    cudaStreamSynchronize(w->stream);
    cudaFree(w->pool);
    w->pool = np;
    w->cap_pool = c;
    return 0;
}

int ensure_small(rp3dg_world* w, size_t n) { return dev_grow(&w->d_small, &w->cap_small, n) ? wfail(w, RP3DG_ENOMEM, "cudaMalloc(small)") : 0; }

// Device rows follow the host's component order: permute them when a sleep,
// wake or type change moved components since the last step.
int sync_rows(rp3dg_world* w) {
    if (w->dev_body_at != w->bcomp.at) {
        const uint32_t n = w->nb;
        std::vector<int32_t> perm(n), inv(n);
        for (uint32_t r = 0; r < n; r++) inv[size_t(w->dev_body_at[r])] = int32_t(r);
        for (uint32_t r = 0; r < n; r++) perm[r] = inv[size_t(w->bcomp.at[r])];
        if (ensure_small(w, n)) return RP3DG_ENOMEM;
        cudaMemcpyAsync(w->d_small, perm.data(), n * 4, cudaMemcpyHostToDevice, w->stream);
        PermArgs a{};
        a.n = n;
        a.perm = w->d_small;
        const int s = w->cur_b, d = 1 - s;
        for (int c = 0; c < BC_NCOL; c++) a.col[a.ncol++] = PermCol{w->bcol[s][c], w->bcol[d][c], 1};
        a.col[a.ncol++] = PermCol{w->biiw[s], w->biiw[d], 3};
        world_permute<<<blocks(n), 128, 0, w->stream>>>(a);
        w->cur_b = d;
        cudaStreamSynchronize(w->stream);
        w->dev_body_at = w->bcomp.at;
        w->tables_dirty = true;
    }
    if (w->dev_col_at != w->ccomp.at) {
        const uint32_t n = w->nc;
        std::vector<int32_t> perm(n), inv(n);
        for (uint32_t r = 0; r < n; r++) inv[size_t(w->dev_col_at[r])] = int32_t(r);
        for (uint32_t r = 0; r < n; r++) perm[r] = inv[size_t(w->ccomp.at[r])];
        if (ensure_small(w, n)) return RP3DG_ENOMEM;
        cudaMemcpyAsync(w->d_small, perm.data(), n * 4, cudaMemcpyHostToDevice, w->stream);
        PermArgs a{};
        a.n = n;
        a.perm = w->d_small;
        const int s = w->cur_c, d = 1 - s;
        for (int c = 0; c < CC_NCOL; c++) a.col[a.ncol++] = PermCol{w->ccol[s][c], w->ccol[d][c], 1};
        world_permute<<<blocks(n), 128, 0, w->stream>>>(a);
        w->cur_c = d;
        cudaStreamSynchronize(w->stream);
        w->dev_col_at = w->ccomp.at;
        w->tables_dirty = true;
    }
    return 0;
}

// The per-row tables that are not float4 columns (gravity flag, collider body
// row, shape, category, mask) are uploaded from host copies whenever the
// component order changed.
int upload_tables(rp3dg_world* w) {
    if (!w->tables_dirty) return 0;
    w->tables_dirty = false;
    std::vector<uint8_t> g(w->nb);
    for (uint32_t r = 0; r < w->nb; r++) g[r] = w->gravity[size_t(w->bcomp.at[r])];
    std::vector<int32_t> cb(w->nc), cs(w->nc);
    std::vector<uint16_t> cat(w->nc), mask(w->nc);
    for (uint32_t r = 0; r < w->nc; r++) {
        const ColliderH& C = w->colliders[size_t(w->ccomp.at[r])];
        cb[r] = w->bcomp.slot[size_t(C.body)];
        cs[r] = C.shape;
        cat[r] = C.category;
        mask[r] = C.mask;
    }
    cudaMemcpyAsync(w->bgrav, g.data(), w->nb, cudaMemcpyHostToDevice, w->stream);
    cudaMemcpyAsync(w->c_body, cb.data(), size_t(w->nc) * 4, cudaMemcpyHostToDevice, w->stream);
    cudaMemcpyAsync(w->c_shape, cs.data(), size_t(w->nc) * 4, cudaMemcpyHostToDevice, w->stream);
    cudaMemcpyAsync(w->c_cat, cat.data(), size_t(w->nc) * 2, cudaMemcpyHostToDevice, w->stream);
    cudaMemcpyAsync(w->c_mask, mask.data(), size_t(w->nc) * 2, cudaMemcpyHostToDevice, w->stream);
    return cudaStreamSynchronize(w->stream) == cudaSuccess ? 0 : wfail(w, RP3DG_ECUDA, "table upload");
}

}  // namespace

extern "C" {

int rp3dg_world_create(rp3dg_ctx* ctx, const rp3dg_world_settings* s, const rp3dg_body_desc* bd, uint32_t nb,
                       const rp3dg_collider_desc* cd, uint32_t nc, rp3dg_world** out) {
    if (!ctx || !s || !out || (nb && !bd) || (nc && !cd)) return ctx ? cfail(ctx, RP3DG_EINVAL, "null argument") : RP3DG_EINVAL;
    *out = nullptr;
    // shape table (host copy)
    auto* w = new rp3dg_world();
    w->ctx = ctx;
    w->stream = static_cast<cudaStream_t>(rp3dg_stream(ctx));
    w->set = *s;
    w->nb = nb;
    w->nc = nc;
    if (rp3dg::get_shapes_host(ctx, &w->shapes) || w->shapes.empty()) {
        delete w;
        return cfail(ctx, RP3DG_EINVAL, "no shape table (rp3dg_set_shapes)");
    }
    for (uint32_t i = 0; i < nc; i++) {
        if (cd[i].body < 0 || uint32_t(cd[i].body) >= nb || (i && cd[i].body < cd[i - 1].body)) {
            delete w;
            return cfail(ctx, RP3DG_EINVAL, "colliders must be grouped by body, bodies ascending");
        }
        if (cd[i].shape < 0 || size_t(cd[i].shape) >= w->shapes.size()) {
            delete w;
            return cfail(ctx, RP3DG_EINVAL, "collider shape outside the shape table");
        }
    }
    for (uint32_t i = 0; i < nb; i++)
        if (bd[i].type < RP3DG_BODY_STATIC || bd[i].type > RP3DG_BODY_DYNAMIC) {
            delete w;
            return cfail(ctx, RP3DG_EINVAL, "bad body type");
        }
    w->bodies.resize(nb);
    w->colliders.resize(nc);
    w->bcomp.reserve_ids(nb);
    w->ccomp.reserve_ids(nc);
    // host-side component data by id
    std::vector<float4> col[BC_NCOL];
    for (auto& v : col) v.assign(nb, make_float4(0.f, 0.f, 0.f, 0.f));
    std::vector<uint8_t> dynamic(nb, 0), gravity(nb, 1);
    std::vector<float4> ccols[CC_NCOL];
    for (auto& v : ccols) v.assign(nc, make_float4(0.f, 0.f, 0.f, 0.f));
    // replay the creation protocol on the component order (the tree comes
    // after the fat AABBs are computed on the device, in the same order)
    uint32_t ci = 0;
    std::vector<int> creation_order;  // colliders in addCollider order
    for (uint32_t b = 0; b < nb; b++) {
        const rp3dg_body_desc& d = bd[b];
        BodyH& B = w->bodies[b];
        w->bcomp.add(int(b), false);  // createRigidBody: enabled, DYNAMIC
        col[BC_POS][b] = make_float4(d.position[0], d.position[1], d.position[2], 0.f);
        col[BC_ORI][b] = make_float4(d.orientation[0], d.orientation[1], d.orientation[2], d.orientation[3]);
        col[BC_MASS][b] = make_float4(1.0f, 1.0f, 0.0f, 0.0f);
        col[BC_IIL][b] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        col[BC_LLOCK][b] = make_float4(1.f, 1.f, 1.f, 0.f);
        col[BC_ALOCK][b] = make_float4(1.f, 1.f, 1.f, 0.f);
        std::vector<uint32_t> mine;
        while (ci < nc && uint32_t(cd[ci].body) == b) {
            const rp3dg_collider_desc& c = cd[ci];
            ColliderH& C = w->colliders[ci];
            C.body = int(b);
            C.shape = c.shape;
            C.category = c.category;
            C.mask = c.mask;
            w->ccomp.add(int(ci), !w->bcomp.enabled(int(b)));
            B.colliders.push_back(int(ci));
            B.has_sim_collider = true;
            ccols[CC_LPOS][ci] = make_float4(c.position[0], c.position[1], c.position[2], 0.f);
            ccols[CC_LORI][ci] = make_float4(c.orientation[0], c.orientation[1], c.orientation[2], c.orientation[3]);
            // Material::mFrictionCoefficientSqrt = sqrt(friction) (Material.h)
            ccols[CC_MAT][ci] = make_float4(std::sqrt(c.friction), c.bounciness, 0.f, 0.f);
            creation_order.push_back(int(ci));
            mine.push_back(ci);
            ci++;
        }
        if (d.type == RP3DG_BODY_DYNAMIC) {
            // updateMassPropertiesFromColliders (RigidBody.cpp:548-608)
            float total = 0.0f, com[3] = {0.f, 0.f, 0.f};
            for (uint32_t k : mine) {
                float vol, in[3], m;
                if (!shape_mass(w->shapes[size_t(cd[k].shape)], cd[k].mass_density, &vol, in, &m)) {
                    delete w;
                    return cfail(ctx, RP3DG_EINVAL, "mass properties of a convex-mesh collider are not supported");
                }
                total += m;
                for (int a = 0; a < 3; a++) com[a] += m * cd[k].position[a];
            }
            if (total > 0.0f)
                for (int a = 0; a < 3; a++) com[a] /= total;
            float tmp[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
            float total2 = 0.0f;
            for (uint32_t k : mine) {
                float vol, in[3], m;
                shape_mass(w->shapes[size_t(cd[k].shape)], cd[k].mass_density, &vol, in, &m);
                total2 += m;
                float R[3][3], RT[3][3], I[3][3];
                quat_matrix(cd[k].orientation, R);
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) RT[r][c] = R[c][r];
                for (int c = 0; c < 3; c++) { RT[0][c] *= in[0]; RT[1][c] *= in[1]; RT[2][c] *= in[2]; }
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) I[r][c] = R[r][0] * RT[0][c] + R[r][1] * RT[1][c] + R[r][2] * RT[2][c];
                const float off[3] = {cd[k].position[0] - com[0], cd[k].position[1] - com[1], cd[k].position[2] - com[2]};
                const float osq = off[0] * off[0] + off[1] * off[1] + off[2] * off[2];
                float O[3][3] = {{osq, 0.f, 0.f}, {0.f, osq, 0.f}, {0.f, 0.f, osq}};
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) O[r][c] += -off[r] * off[c];
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) O[r][c] *= m;
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) tmp[r][c] += I[r][c] + O[r][c];
            }
            const float in[3] = {tmp[0][0], tmp[1][1], tmp[2][2]};
            col[BC_COML][b] = make_float4(com[0], com[1], com[2], 0.f);
            col[BC_IIL][b] = make_float4(in[0] != 0.0f ? 1.0f / in[0] : 0.0f, in[1] != 0.0f ? 1.0f / in[1] : 0.0f,
                                         in[2] != 0.0f ? 1.0f / in[2] : 0.0f, 0.f);
            col[BC_MASS][b].x = total2;
            col[BC_MASS][b].y = total2 > 0.0f ? 1.0f / total2 : 0.0f;
            dynamic[b] = 1;
        } else {
            // setType (RigidBody.cpp:66-130)
            col[BC_MASS][b].y = 0.0f;
            col[BC_IIL][b] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (d.type == RP3DG_BODY_STATIC) set_body_disabled(w, int(b), true);
        }
        B.type = d.type;
        col[BC_MASS][b].z = d.linear_damping;
        col[BC_MASS][b].w = d.angular_damping;
        col[BC_LLOCK][b] = make_float4(d.linear_lock[0], d.linear_lock[1], d.linear_lock[2], 0.f);
        col[BC_ALOCK][b] = make_float4(d.angular_lock[0], d.angular_lock[1], d.angular_lock[2], 0.f);
        gravity[b] = d.gravity_enabled ? 1 : 0;
        B.allowed_sleep = d.allowed_to_sleep != 0;
        if (d.type != RP3DG_BODY_STATIC) {
            col[BC_LV][b] = make_float4(d.linear_velocity[0], d.linear_velocity[1], d.linear_velocity[2], 0.f);
            col[BC_AV][b] = make_float4(d.angular_velocity[0], d.angular_velocity[1], d.angular_velocity[2], 0.f);
        }
    }
    w->gravity = gravity;
    // device arrays in component order
    cudaError_t e = cudaSuccess;
    auto M = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 16)); };
    for (int k = 0; k < 2; k++) {
        for (int c = 0; c < BC_NCOL; c++) M((void**)&w->bcol[k][c], size_t(nb) * 16);
        M((void**)&w->biiw[k], size_t(nb) * 48);
        for (int c = 0; c < CC_NCOL; c++) M((void**)&w->ccol[k][c], size_t(nc) * 16);
    }
    M((void**)&w->bgrav, nb);
    M((void**)&w->c_body, size_t(nc) * 4);
    M((void**)&w->c_shape, size_t(nc) * 4);
    M((void**)&w->c_cat, size_t(nc) * 2);
    M((void**)&w->c_mask, size_t(nc) * 2);
    M((void**)&w->c_moved, nc);
    if (e != cudaSuccess) {
        rp3dg_world_destroy(w);
        return cfail(ctx, RP3DG_ENOMEM, "cudaMalloc(world)");
    }
    w->dev_body_at = w->bcomp.at;
    w->dev_col_at = w->ccomp.at;
    {
        std::vector<float4> tmp(std::max(nb, nc));
        for (int c = 0; c < BC_NCOL; c++) {
            for (uint32_t r = 0; r < nb; r++) tmp[r] = col[c][size_t(w->bcomp.at[r])];
            cudaMemcpyAsync(w->bcol[0][c], tmp.data(), size_t(nb) * 16, cudaMemcpyHostToDevice, w->stream);
            cudaStreamSynchronize(w->stream);
        }
        cudaMemsetAsync(w->biiw[0], 0, size_t(nb) * 48, w->stream);
        for (int c = 0; c < CC_NCOL; c++) {
            for (uint32_t r = 0; r < nc; r++) tmp[r] = ccols[c][size_t(w->ccomp.at[r])];
            cudaMemcpyAsync(w->ccol[0][c], tmp.data(), size_t(nc) * 16, cudaMemcpyHostToDevice, w->stream);
            cudaStreamSynchronize(w->stream);
        }
        std::vector<uint8_t> dyn(nb);
        for (uint32_t r = 0; r < nb; r++) dyn[r] = dynamic[size_t(w->bcomp.at[r])];
        uint8_t* d_dyn = nullptr;
        cudaMalloc(&d_dyn, std::max<uint32_t>(nb, 1));
        cudaMemcpyAsync(d_dyn, dyn.data(), nb, cudaMemcpyHostToDevice, w->stream);
        w->tables_dirty = true;
        int rc = upload_tables(w);
        if (rc) { cudaFree(d_dyn); rp3dg_world_destroy(w); return rc; }
        const uint32_t n = std::max(nb, nc);
        if (n)
            world_setup<<<blocks(n), 128, 0, w->stream>>>(nb, w->bcol[0][BC_POS], w->bcol[0][BC_ORI], w->bcol[0][BC_COML],
                                                          w->bcol[0][BC_COMW], d_dyn, nc, w->c_body, w->ccol[0][CC_LPOS],
                                                          w->ccol[0][CC_LORI], w->ccol[0][CC_WPOS], w->ccol[0][CC_WORI]);
        cudaStreamSynchronize(w->stream);
        cudaFree(d_dyn);
    }
    // initial fat AABBs of every collider (addCollider -> addObject)
    if (nc) {
        uint8_t* force = nullptr;
        cudaMalloc(&force, nc);
        cudaMemsetAsync(force, 1, nc, w->stream);
        rp3dg_broadphase bp{};
        bp.n = nc;
        bp.n_update = nc;
        bp.shape = w->c_shape;
        bp.body = w->c_body;
        bp.world_position = reinterpret_cast<rp3dg_float4*>(w->ccol[0][CC_WPOS]);
        bp.world_orientation = reinterpret_cast<rp3dg_float4*>(w->ccol[0][CC_WORI]);
        bp.force_reinsert = force;
        bp.fat_min = reinterpret_cast<rp3dg_float4*>(w->ccol[0][CC_FMIN]);
        bp.fat_max = reinterpret_cast<rp3dg_float4*>(w->ccol[0][CC_FMAX]);
        bp.moved = w->c_moved;
        int rc = rp3dg_broadphase_update_device(ctx, &bp);
        std::vector<float4> fmin(nc), fmax(nc);
        cudaMemcpyAsync(fmin.data(), w->ccol[0][CC_FMIN], size_t(nc) * 16, cudaMemcpyDeviceToHost, w->stream);
        cudaMemcpyAsync(fmax.data(), w->ccol[0][CC_FMAX], size_t(nc) * 16, cudaMemcpyDeviceToHost, w->stream);
        e = cudaStreamSynchronize(w->stream);
        cudaFree(force);
        if (rc || e != cudaSuccess) {
            rp3dg_world_destroy(w);
            return rc ? rc : cfail(ctx, RP3DG_ECUDA, "initial broad phase");
        }
        w->bp_to_collider.clear();
        for (int c : creation_order) {
            const uint32_t r = uint32_t(w->ccomp.slot[size_t(c)]);
            Box box;
            box.mn[0] = fmin[r].x; box.mn[1] = fmin[r].y; box.mn[2] = fmin[r].z;
            box.mx[0] = fmax[r].x; box.mx[1] = fmax[r].y; box.mx[2] = fmax[r].z;
            const int id = w->tree.add_object(box, c);
            w->colliders[size_t(c)].bp = id;
            if (size_t(id) >= w->bp_to_collider.size()) w->bp_to_collider.resize(size_t(id) + 1, -1);
            w->bp_to_collider[size_t(id)] = c;
            w->moved.add(id);
        }
    }
    *out = w;
    return 0;
}

void rp3dg_world_destroy(rp3dg_world* w) {
    if (!w) return;
    for (int k = 0; k < 2; k++) {
        for (int c = 0; c < BC_NCOL; c++) cudaFree(w->bcol[k][c]);
        cudaFree(w->biiw[k]);
        for (int c = 0; c < CC_NCOL; c++) cudaFree(w->ccol[k][c]);
        w->cbuf[k].release();
    }
    cudaFree(w->bgrav); cudaFree(w->c_body); cudaFree(w->c_shape); cudaFree(w->c_cat); cudaFree(w->c_mask);
    cudaFree(w->c_moved); cudaFree(w->pool); cudaFree(w->d_small);
    cudaFree(w->d_items); cudaFree(w->d_s1); cudaFree(w->d_s2); cudaFree(w->d_p1); cudaFree(w->d_r1);
    cudaFree(w->d_p2); cudaFree(w->d_r2); cudaFree(w->d_rep); cudaFree(w->d_coll); cudaFree(w->d_nct);
    cudaFree(w->d_cache); cudaFree(w->d_nd); cudaFree(w->d_l1); cudaFree(w->d_l2);
    cudaFree(w->d_mids); cudaFree(w->d_msrc); cudaFree(w->d_mprev); cudaFree(w->d_istart); cudaFree(w->d_icount);
    cudaFreeHost(w->h_items); cudaFreeHost(w->h_out); cudaFreeHost(w->h_mids); cudaFreeHost(w->h_msrc);
    cudaFreeHost(w->h_mprev); cudaFreeHost(w->h_istart); cudaFreeHost(w->h_icount); cudaFreeHost(w->h_step);
    delete w;
}

int rp3dg_world_update(rp3dg_world* w, float dt) {
    if (!w) return RP3DG_EINVAL;
    if (!(dt > 0.0f)) return wfail(w, RP3DG_EINVAL, "dt must be positive");
    cudaStream_t st = w->stream;
    rp3dg_ctx* ctx = w->ctx;
    std::memset(&w->stats, 0, sizeof(w->stats));
    // phase timer: with profiling on, the stream is drained at each mark so
    // that GPU time is charged to the phase that queued it
    auto mark = [&](int k) {
        if (!w->profiling) return;
        cudaStreamSynchronize(w->stream);
        const auto now = std::chrono::steady_clock::now();
        w->phase_ms[k] += std::chrono::duration<double, std::milli>(now - w->t_mark).count();
        w->t_mark = now;
    };
    if (w->profiling) w->t_mark = std::chrono::steady_clock::now();

    // ---- computeCollisionDetection: broad phase (host order, GPU fat AABBs)
    broad_phase(w);
    mark(0);

    // ---- middle phase: narrow-phase batches in pair-array order
    std::vector<int4> by_algo[NB_ALGOS];
    std::vector<uint32_t> pair_of[NB_ALGOS];
    for (uint32_t i = 0; i < w->pairs.size(); i++) {
        PairH& p = w->pairs[i];
        p.coll_curr = false;
        const bool e1 = w->ccomp.enabled(p.c1), e2 = w->ccomp.enabled(p.c2);
        if (!(e1 || e2)) continue;
        const int a = p.algo - 1;
        by_algo[a].push_back(make_int4(w->ccomp.slot[size_t(p.c1)], w->ccomp.slot[size_t(p.c2)], p.cache, 1));
        pair_of[a].push_back(i);
    }
    w->items.clear();
    w->item_pair.clear();
    for (int a = 0; a < NB_ALGOS; a++) {
        w->batch_start[a] = uint32_t(w->items.size());
        w->items.insert(w->items.end(), by_algo[a].begin(), by_algo[a].end());
        w->item_pair.insert(w->item_pair.end(), pair_of[a].begin(), pair_of[a].end());
    }
    w->batch_start[NB_ALGOS] = uint32_t(w->items.size());
    const uint32_t T = uint32_t(w->items.size());
    w->stats.narrowphase_tests = T;
    w->stats.overlapping_pairs = uint32_t(w->pairs.size());

    mark(1);
    int rc = ensure_pool(w);
    if (rc) return rc;
    if (!w->reset_slots.empty()) {
        if (ensure_small(w, w->reset_slots.size())) return RP3DG_ENOMEM;
        cudaMemcpyAsync(w->d_small, w->reset_slots.data(), w->reset_slots.size() * 4, cudaMemcpyHostToDevice, st);
        world_reset_cache<<<blocks(uint32_t(w->reset_slots.size())), 128, 0, st>>>(uint32_t(w->reset_slots.size()),
                                                                                 w->d_small, w->pool);
        w->reset_slots.clear();
    }
    rc = sync_rows(w);
    if (rc) return rc;
    rc = upload_tables(w);
    if (rc) return rc;
    const int cb = w->cur_b, cc = w->cur_c;

    w->cpairs.clear();
    if (T) {
        rc = ensure_items(w, T);
        if (rc) return rc;
        std::memcpy(w->h_items, w->items.data(), size_t(T) * 16);
        cudaMemcpyAsync(w->d_items, w->h_items, size_t(T) * 16, cudaMemcpyHostToDevice, st);
        GatherArgs g;
        g.n = T;
        g.items = w->d_items;
        g.c_shape = w->c_shape;
        g.c_wpos = w->ccol[cc][CC_WPOS];
        g.c_wori = w->ccol[cc][CC_WORI];
        g.pool = w->pool;
        g.s1 = w->d_s1; g.s2 = w->d_s2;
        g.p1 = w->d_p1; g.r1 = w->d_r1; g.p2 = w->d_p2; g.r2 = w->d_r2;
        g.report = w->d_rep;
        g.cache = w->d_cache;
        world_gather_batch<<<blocks(T), 128, 0, st>>>(g);
        // ---- narrow phase + manifold step, one call per algorithm batch
        for (int a = 0; a < NB_ALGOS; a++) {
            const uint32_t s0 = w->batch_start[a], n = w->batch_start[a + 1] - s0;
            if (!n) continue;
            rp3dg_pair_batch pb{};
            pb.n = n;
            pb.shape1 = w->d_s1 + s0; pb.shape2 = w->d_s2 + s0;
            pb.pos1 = reinterpret_cast<rp3dg_float4*>(w->d_p1 + s0);
            pb.rot1 = reinterpret_cast<rp3dg_float4*>(w->d_r1 + s0);
            pb.pos2 = reinterpret_cast<rp3dg_float4*>(w->d_p2 + s0);
            pb.rot2 = reinterpret_cast<rp3dg_float4*>(w->d_r2 + s0);
            pb.report_contacts = w->d_rep + s0;
            pb.cache = w->d_cache + s0;
            rp3dg_contact_batch cbt{};
            cbt.is_colliding = w->d_coll + s0;
            cbt.nb_contacts = w->d_nct + s0;
            cbt.normal_depth = reinterpret_cast<rp3dg_float4*>(w->d_nd + size_t(s0) * MAXC);
            cbt.local1 = reinterpret_cast<rp3dg_float4*>(w->d_l1 + size_t(s0) * MAXC);
            cbt.local2 = reinterpret_cast<rp3dg_float4*>(w->d_l2 + size_t(s0) * MAXC);
            cbt.max_contacts = MAXC;
            rc = rp3dg_narrowphase_device(ctx, a + 1, &pb, &cbt, 1);
            if (rc) return wfail(w, rc, std::string("narrow phase: ") + rp3dg_last_error(ctx));
            rc = rp3dg_reduce_contacts_device(ctx, &pb, &cbt, nullptr);
            if (rc) return wfail(w, rc, std::string("manifold step: ") + rp3dg_last_error(ctx));
        }
        world_scatter_cache<<<blocks(T), 128, 0, st>>>(T, w->d_items, w->d_cache, w->pool);
        cudaMemcpyAsync(w->h_out, w->d_coll, T, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(w->h_out + T, w->d_nct, T, cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return wcuda(w, e, "narrow phase");
        // ---- processAllPotentialContacts: contact pairs in batch order
        for (uint32_t it = 0; it < T; it++) {
            if (!w->h_out[it]) continue;
            PairH& p = w->pairs[w->item_pair[it]];
            p.coll_curr = true;
            ContactPairH c;
            c.id = p.id;
            c.c1 = p.c1;
            c.c2 = p.c2;
            c.b1 = w->colliders[size_t(p.c1)].body;
            c.b2 = w->colliders[size_t(p.c2)].body;
            c.item = it;
            c.k = w->h_out[T + it];
            w->cpairs.push_back(c);
        }
    }
    mark(2);
    // addContactPairsToBodies
    for (uint32_t p = 0; p < w->cpairs.size(); p++) {
        w->bodies[size_t(w->cpairs[p].b1)].contact_pairs.push_back(p);
        w->bodies[size_t(w->cpairs[p].b2)].contact_pairs.push_back(p);
    }
    w->stats.contact_pairs = uint32_t(w->cpairs.size());

    // ---- createIslands (PhysicsWorld.cpp:695-866)
    std::vector<int32_t> zero_rows;
    w->island_order.clear();
    w->islands.clear();
    for (auto& B : w->bodies) B.in_island = false;
    {
        uint32_t total_manifolds = 0;
        std::vector<int> stack, statics;
        for (uint32_t s = 0; s < w->bcomp.n_enabled; s++) {
            const int b0 = w->bcomp.at[s];
            if (w->bodies[size_t(b0)].in_island) continue;
            if (w->bodies[size_t(b0)].type == RP3DG_BODY_STATIC) continue;
            stack.clear();
            w->bodies[size_t(b0)].in_island = true;
            stack.push_back(b0);
            IslandH isl;
            isl.manifold_start = total_manifolds;
            const size_t isl_index = w->islands.size();
            w->islands.push_back(isl);
            while (!stack.empty()) {
                const int b = stack.back();
                stack.pop_back();
                w->islands[isl_index].bodies.push_back(b);
                set_sleeping(w, b, false, &zero_rows);
                if (w->bodies[size_t(b)].type == RP3DG_BODY_STATIC) {
                    statics.push_back(b);
                    continue;
                }
                for (uint32_t cpi : w->bodies[size_t(b)].contact_pairs) {
                    ContactPairH& cp = w->cpairs[cpi];
                    if (cp.in_island) continue;
                    cp.in_island = true;
                    const int other = cp.b1 == b ? cp.b2 : cp.b1;
                    if (w->bodies[size_t(other)].has_sim_collider) {
                        w->island_order.push_back(cpi);
                        total_manifolds += 1;
                        w->islands[isl_index].manifold_count += 1;
                        if (w->bodies[size_t(other)].in_island) continue;
                        stack.push_back(other);
                        w->bodies[size_t(other)].in_island = true;
                    }
                }
            }
            for (int sb : statics) w->bodies[size_t(sb)].in_island = false;
            statics.clear();
        }
        for (auto& cp : w->cpairs) {
            w->bodies[size_t(cp.b1)].contact_pairs.clear();
            w->bodies[size_t(cp.b2)].contact_pairs.clear();
        }
    }
    w->stats.islands = uint32_t(w->islands.size());

    mark(3);
    // ---- createContacts: manifolds and points in island order
    rc = sync_rows(w);
    if (rc) return rc;
    rc = upload_tables(w);
    if (rc) return rc;
    const int bc = w->cur_b, ccur = w->cur_c;
    ContactBuf& CB = w->cbuf[w->cur_cb];
    ContactBuf& PB = w->cbuf[1 - w->cur_cb];
    const uint32_t nm = uint32_t(w->island_order.size());
    uint32_t np = 0;
    {
        if (dev_grow(&w->d_mids, &w->cap_m, std::max<uint32_t>(nm, 1))) return wfail(w, RP3DG_ENOMEM, "cudaMalloc");
        if (w->cap_hm < nm || !w->h_mids) {
            size_t cap = std::max<size_t>(nm, 64);
            cudaFreeHost(w->h_mids); cudaFreeHost(w->h_msrc); cudaFreeHost(w->h_mprev);
            cudaFree(w->d_msrc); cudaFree(w->d_mprev);
            cudaFree(w->d_mids);
            w->cap_m = 0;
            if (cudaMallocHost(&w->h_mids, cap * 16) || cudaMallocHost(&w->h_msrc, cap * 16) ||
                cudaMallocHost(&w->h_mprev, cap * 16) || cudaMalloc(&w->d_mids, cap * 16) ||
                cudaMalloc(&w->d_msrc, cap * 16) || cudaMalloc(&w->d_mprev, cap * 16))
                return wfail(w, RP3DG_ENOMEM, "allocation of manifold staging");
            w->cap_hm = cap;
            w->cap_m = cap;
        }
        for (uint32_t m = 0; m < nm; m++) {
            ContactPairH& cp = w->cpairs[w->island_order[m]];
            cp.manifold = m;
            cp.point = np;
            uint32_t a = 0;
            while (cp.item >= w->batch_start[a + 1]) a++;
            const uint32_t s0 = w->batch_start[a];
            w->h_mids[m] = make_int4(w->bcomp.slot[size_t(cp.b1)], w->bcomp.slot[size_t(cp.b2)],
                                     w->ccomp.slot[size_t(cp.c1)], w->ccomp.slot[size_t(cp.c2)]);
            w->h_msrc[m] = make_int4(int(cp.item - s0), int(w->batch_start[a + 1] - s0), int(s0), int(np));
            auto it = w->prev_map.find(cp.id);
            if (it != w->prev_map.end() && w->prev_cpairs[it->second].in_island) {
                const ContactPairH& pc = w->prev_cpairs[it->second];
                w->h_mprev[m] = make_int4(int(pc.manifold), 1, int(pc.point), int(pc.k));
            } else {
                w->h_mprev[m] = make_int4(-1, 0, 0, 0);
            }
            np += cp.k;
        }
        if (CB.ensure(std::max<uint32_t>(nm, 1), std::max<uint32_t>(np, 1))) return wfail(w, RP3DG_ENOMEM, "cudaMalloc(contacts)");
        if (nm) {
            cudaMemcpyAsync(w->d_mids, w->h_mids, size_t(nm) * 16, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(w->d_msrc, w->h_msrc, size_t(nm) * 16, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(w->d_mprev, w->h_mprev, size_t(nm) * 16, cudaMemcpyHostToDevice, st);
            PackArgs a;
            a.nm = nm;
            a.ids = w->d_mids;
            a.src = w->d_msrc;
            a.prev = w->d_mprev;
            a.kept_count = w->d_nct;
            a.b_nd = w->d_nd; a.b_l1 = w->d_l1; a.b_l2 = w->d_l2;
            a.cos_similar = w->set.cos_angle_similar_contact_manifold;
            a.persist2 = w->set.persistent_contact_distance_threshold * w->set.persistent_contact_distance_threshold;
            a.pm_pstart = PB.pstart; a.pm_fv1 = PB.fv1; a.pm_fv2 = PB.fv2; a.pm_fimp = PB.fimp;
            a.pp_nd = PB.nd; a.pp_l1 = PB.l1; a.pp_imp = PB.imp; a.pp_rest = PB.rest;
            a.m_ids = CB.ids; a.m_pstart = CB.pstart; a.m_npts = CB.npts;
            a.m_fv1 = CB.fv1; a.m_fv2 = CB.fv2; a.m_fimp = CB.fimp;
            a.p_nd = CB.nd; a.p_l1 = CB.l1; a.p_l2 = CB.l2; a.p_imp = CB.imp; a.p_rest = CB.rest;
            world_pack_contacts<<<blocks(nm), 128, 0, st>>>(a);
        }
    }
    CB.nm = nm;
    CB.np = np;
    w->stats.manifolds = nm;
    w->stats.contact_points = np;
    // computeMapPreviousContactPairs for the next step
    w->prev_map.clear();
    for (uint32_t i = 0; i < w->cpairs.size(); i++) w->prev_map[w->cpairs[i].id] = i;

    // islands as manifold ranges
    const uint32_t ni = uint32_t(w->islands.size());
    if (w->cap_hi < ni || !w->h_istart) {
        size_t cap = std::max<size_t>(ni, 64);
        cudaFreeHost(w->h_istart); cudaFreeHost(w->h_icount); cudaFree(w->d_istart); cudaFree(w->d_icount);
        if (cudaMallocHost(&w->h_istart, cap * 4) || cudaMallocHost(&w->h_icount, cap * 4) ||
            cudaMalloc(&w->d_istart, cap * 4) || cudaMalloc(&w->d_icount, cap * 4))
            return wfail(w, RP3DG_ENOMEM, "allocation of island arrays");
        w->cap_hi = cap;
        w->cap_i = cap;
    }
    for (uint32_t i = 0; i < ni; i++) {
        w->h_istart[i] = w->islands[i].manifold_start;
        w->h_icount[i] = w->islands[i].manifold_count;
    }
    if (ni) {
        cudaMemcpyAsync(w->d_istart, w->h_istart, size_t(ni) * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(w->d_icount, w->h_icount, size_t(ni) * 4, cudaMemcpyHostToDevice, st);
    }

    mark(4);
    // ---- dynamics stage (inertia, velocities, solver, positions, state)
    {
        rp3dg_dynamics_params pr{};
        pr.dt = dt;
        pr.gravity[0] = w->set.gravity[0]; pr.gravity[1] = w->set.gravity[1]; pr.gravity[2] = w->set.gravity[2];
        pr.gravity_enabled = 1;
        pr.velocity_iterations = w->set.velocity_iterations;
        pr.split_impulse = 1;
        pr.restitution_velocity_threshold = w->set.restitution_velocity_threshold;
        rp3dg_bodies B{};
        B.n = w->nb;
        B.n_enabled = w->bcomp.n_enabled;
        auto F = [](float4* p) { return reinterpret_cast<rp3dg_float4*>(p); };
        B.position = F(w->bcol[bc][BC_POS]); B.orientation = F(w->bcol[bc][BC_ORI]);
        B.com_world = F(w->bcol[bc][BC_COMW]); B.com_local = F(w->bcol[bc][BC_COML]);
        B.linear_velocity = F(w->bcol[bc][BC_LV]); B.angular_velocity = F(w->bcol[bc][BC_AV]);
        B.force = F(w->bcol[bc][BC_F]); B.torque = F(w->bcol[bc][BC_T]);
        B.inv_inertia_local = F(w->bcol[bc][BC_IIL]); B.inv_inertia_world = F(w->biiw[bc]);
        B.mass = F(w->bcol[bc][BC_MASS]); B.linear_lock = F(w->bcol[bc][BC_LLOCK]); B.angular_lock = F(w->bcol[bc][BC_ALOCK]);
        B.gravity = w->bgrav;
        rp3dg_colliders C{};
        C.n = w->nc;
        C.n_enabled = w->ccomp.n_enabled;
        C.body = w->c_body;
        C.local_position = F(w->ccol[ccur][CC_LPOS]); C.local_orientation = F(w->ccol[ccur][CC_LORI]);
        C.world_position = F(w->ccol[ccur][CC_WPOS]); C.world_orientation = F(w->ccol[ccur][CC_WORI]);
        C.material = F(w->ccol[ccur][CC_MAT]);
        rp3dg_manifolds Mf{};
        Mf.n = nm;
        Mf.ids = reinterpret_cast<int32_t*>(CB.ids);
        Mf.point_start = CB.pstart; Mf.nb_points = CB.npts;
        Mf.friction_vector1 = F(CB.fv1); Mf.friction_vector2 = F(CB.fv2); Mf.friction_impulse = F(CB.fimp);
        rp3dg_points P{};
        P.n = np;
        P.normal_depth = F(CB.nd); P.local1 = F(CB.l1); P.local2 = F(CB.l2);
        P.penetration_impulse = CB.imp; P.is_resting = CB.rest;
        rp3dg_islands I{};
        I.n = ni;
        I.manifold_start = w->d_istart;
        I.manifold_count = w->d_icount;
        rc = rp3dg_dynamics_step_device(ctx, &pr, &B, &C, &Mf, &P, &I);
        if (rc) return wfail(w, rc, std::string("dynamics: ") + rp3dg_last_error(ctx));
    }

    mark(5);
    // ---- updateColliders: world AABBs, fat-AABB test, reinsertion flags
    const uint32_t ncu = w->ccomp.n_enabled, nbe = w->bcomp.n_enabled;
    const size_t step_bytes = size_t(ncu) + size_t(ncu) * 32 + size_t(nbe) * 32 + 64;
    if (host_grow(&w->h_step, &w->cap_hstep, step_bytes)) return wfail(w, RP3DG_ENOMEM, "cudaMallocHost(step)");
    uint8_t* h_moved = w->h_step;
    float4* h_fmin = reinterpret_cast<float4*>(w->h_step + ((size_t(ncu) + 15) & ~size_t(15)));
    float4* h_fmax = h_fmin + ncu;
    float4* h_lv = h_fmax + ncu;
    float4* h_av = h_lv + nbe;
    if (ncu) {
        rp3dg_broadphase bp{};
        bp.n = w->nc;
        bp.n_update = ncu;
        bp.shape = w->c_shape;
        bp.body = w->c_body;
        bp.world_position = reinterpret_cast<rp3dg_float4*>(w->ccol[ccur][CC_WPOS]);
        bp.world_orientation = reinterpret_cast<rp3dg_float4*>(w->ccol[ccur][CC_WORI]);
        bp.fat_min = reinterpret_cast<rp3dg_float4*>(w->ccol[ccur][CC_FMIN]);
        bp.fat_max = reinterpret_cast<rp3dg_float4*>(w->ccol[ccur][CC_FMAX]);
        bp.moved = w->c_moved;
        rc = rp3dg_broadphase_update_device(ctx, &bp);
        if (rc) return wfail(w, rc, std::string("broad-phase update: ") + rp3dg_last_error(ctx));
        cudaMemcpyAsync(h_moved, w->c_moved, ncu, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(h_fmin, w->ccol[ccur][CC_FMIN], size_t(ncu) * 16, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(h_fmax, w->ccol[ccur][CC_FMAX], size_t(ncu) * 16, cudaMemcpyDeviceToHost, st);
    }
    if (w->set.sleeping_enabled && nbe) {
        cudaMemcpyAsync(h_lv, w->bcol[bc][BC_LV], size_t(nbe) * 16, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(h_av, w->bcol[bc][BC_AV], size_t(nbe) * 16, cudaMemcpyDeviceToHost, st);
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return wcuda(w, e, "step");
    uint32_t nmoved = 0;
    for (uint32_t r = 0; r < ncu; r++) {
        if (!h_moved[r]) continue;
        const int c = w->ccomp.at[r];
        Box box;
        box.mn[0] = h_fmin[r].x; box.mn[1] = h_fmin[r].y; box.mn[2] = h_fmin[r].z;
        box.mx[0] = h_fmax[r].x; box.mx[1] = h_fmax[r].y; box.mx[2] = h_fmax[r].z;
        w->tree.reinsert(w->colliders[size_t(c)].bp, box);
        add_moved(w, c);
        nmoved++;
    }
    w->stats.moved_colliders = nmoved;

    mark(6);
    // ---- updateSleepingBodies (PhysicsWorld.cpp:871-926)
    if (w->set.sleeping_enabled) {
        // velocities by body id, read before any body falls asleep
        std::vector<float4> lv(w->nb), av(w->nb);
        for (uint32_t r = 0; r < nbe; r++) {
            lv[size_t(w->bcomp.at[r])] = h_lv[r];
            av[size_t(w->bcomp.at[r])] = h_av[r];
        }
        const float slv2 = w->set.sleep_linear_velocity * w->set.sleep_linear_velocity;
        const float sav2 = w->set.sleep_angular_velocity * w->set.sleep_angular_velocity;
        for (const IslandH& isl : w->islands) {
            float min_sleep = 3.40282347e+38f;
            for (int b : isl.bodies) {
                BodyH& B = w->bodies[size_t(b)];
                if (B.type == RP3DG_BODY_STATIC) continue;
                const float4 l = lv[size_t(b)], a = av[size_t(b)];
                if (l.x * l.x + l.y * l.y + l.z * l.z > slv2 || a.x * a.x + a.y * a.y + a.z * a.z > sav2 ||
                    !B.allowed_sleep) {
                    B.sleep_time = 0.0f;
                    min_sleep = 0.0f;
                } else {
                    B.sleep_time += dt;
                    if (B.sleep_time < min_sleep) min_sleep = B.sleep_time;
                }
            }
            if (min_sleep >= w->set.time_before_sleep)
                for (int b : isl.bodies) set_sleeping(w, b, true, &zero_rows);
        }
    }
    // velocities / forces of bodies put to sleep (rows in the current device order)
    if (!zero_rows.empty()) {
        std::vector<int32_t> rows, row_of(w->nb);
        for (uint32_t r = 0; r < w->nb; r++) row_of[size_t(w->dev_body_at[r])] = int32_t(r);
        for (int b : zero_rows)
            if (w->bodies[size_t(b)].sleeping) rows.push_back(row_of[size_t(b)]);
        if (!rows.empty()) {
            if (ensure_small(w, rows.size())) return RP3DG_ENOMEM;
            cudaMemcpyAsync(w->d_small, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, st);
            world_zero_rows<<<blocks(uint32_t(rows.size())), 128, 0, st>>>(uint32_t(rows.size()), w->d_small,
                                                                           w->bcol[bc][BC_LV], w->bcol[bc][BC_AV],
                                                                           w->bcol[bc][BC_F], w->bcol[bc][BC_T]);
        }
    }
    // resetBodiesForceAndTorque
    cudaMemsetAsync(w->bcol[bc][BC_F], 0, size_t(w->nb) * 16, st);
    cudaMemsetAsync(w->bcol[bc][BC_T], 0, size_t(w->nb) * 16, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return wcuda(w, e, "end of step");
    // collidingInPreviousFrame for the next step (updateCollidingInPreviousFrame
    // runs in reportContactsAndTriggers)
    for (auto& p : w->pairs) p.coll_prev = p.coll_curr;
    w->prev_cpairs.swap(w->cpairs);
    w->cur_cb = 1 - w->cur_cb;
    w->stats.disabled_pairs = uint32_t(w->disabled.size());
    w->stats.enabled_bodies = w->bcomp.n_enabled;
    mark(7);
    return 0;
}

int rp3dg_world_set_profiling(rp3dg_world* w, int enable) {
    if (!w) return RP3DG_EINVAL;
    w->profiling = enable != 0;
    for (double& t : w->phase_ms) t = 0.0;
    return 0;
}

int rp3dg_world_get_phase_times(rp3dg_world* w, double* ms, uint32_t n) {
    if (!w || !ms) return RP3DG_EINVAL;
    for (uint32_t i = 0; i < n && i < 8; i++) ms[i] = w->phase_ms[i];
    return 0;
}

int rp3dg_world_get_bodies(rp3dg_world* w, float* position, float* orientation, float* linear_velocity,
                           float* angular_velocity, uint8_t* sleeping) {
    if (!w) return RP3DG_EINVAL;
    const uint32_t n = w->nb;
    std::vector<float4> p(n), q(n), lv(n), av(n);
    const int b = w->cur_b;
    cudaMemcpyAsync(p.data(), w->bcol[b][BC_POS], size_t(n) * 16, cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(q.data(), w->bcol[b][BC_ORI], size_t(n) * 16, cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(lv.data(), w->bcol[b][BC_LV], size_t(n) * 16, cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(av.data(), w->bcol[b][BC_AV], size_t(n) * 16, cudaMemcpyDeviceToHost, w->stream);
    cudaError_t e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return wcuda(w, e, "read bodies");
    for (uint32_t r = 0; r < n; r++) {
        const size_t id = size_t(w->dev_body_at[r]);
        if (position) { position[3 * id] = p[r].x; position[3 * id + 1] = p[r].y; position[3 * id + 2] = p[r].z; }
        if (orientation) {
            orientation[4 * id] = q[r].x; orientation[4 * id + 1] = q[r].y;
            orientation[4 * id + 2] = q[r].z; orientation[4 * id + 3] = q[r].w;
        }
        if (linear_velocity) {
            linear_velocity[3 * id] = lv[r].x; linear_velocity[3 * id + 1] = lv[r].y; linear_velocity[3 * id + 2] = lv[r].z;
        }
        if (angular_velocity) {
            angular_velocity[3 * id] = av[r].x; angular_velocity[3 * id + 1] = av[r].y; angular_velocity[3 * id + 2] = av[r].z;
        }
        if (sleeping) sleeping[id] = w->bodies[id].sleeping ? 1 : 0;
    }
    return 0;
}

int rp3dg_world_get_pairs(rp3dg_world* w, uint64_t* ids, uint32_t capacity, uint32_t* n) {
    if (!w || !n) return RP3DG_EINVAL;
    uint32_t k = 0;
    for (const auto& p : w->pairs) { if (ids && k < capacity) ids[k] = p.id; k++; }
    for (const auto& p : w->disabled) { if (ids && k < capacity) ids[k] = p.id; k++; }
    *n = k;
    return 0;
}

int rp3dg_world_get_contacts(rp3dg_world* w, int32_t* body1, int32_t* body2, uint8_t* nb_points, uint32_t capacity,
                             float* normal_depth, float* local1, float* local2, uint32_t capacity_points,
                             uint32_t* nb_manifolds, uint32_t* nb_contact_points) {
    if (!w) return RP3DG_EINVAL;
    // the arrays of the last step are the "previous" buffer after the swap
    const ContactBuf& B = w->cbuf[1 - w->cur_cb];
    const std::vector<ContactPairH>& cps = w->prev_cpairs;
    if (nb_manifolds) *nb_manifolds = B.nm;
    if (nb_contact_points) *nb_contact_points = B.np;
    std::vector<uint32_t> order(B.nm);
    for (uint32_t i = 0; i < cps.size(); i++)
        if (cps[i].in_island) order[cps[i].manifold] = i;
    for (uint32_t m = 0; m < B.nm && m < capacity; m++) {
        const ContactPairH& c = cps[order[m]];
        if (body1) body1[m] = c.b1;
        if (body2) body2[m] = c.b2;
        if (nb_points) nb_points[m] = uint8_t(c.k);
    }
    const uint32_t np = std::min(B.np, capacity_points);
    if (np) {
        if (normal_depth) cudaMemcpyAsync(normal_depth, B.nd, size_t(np) * 16, cudaMemcpyDeviceToHost, w->stream);
        if (local1) cudaMemcpyAsync(local1, B.l1, size_t(np) * 16, cudaMemcpyDeviceToHost, w->stream);
        if (local2) cudaMemcpyAsync(local2, B.l2, size_t(np) * 16, cudaMemcpyDeviceToHost, w->stream);
    }
    cudaError_t e = cudaStreamSynchronize(w->stream);
    return e == cudaSuccess ? 0 : wcuda(w, e, "read contacts");
}

int rp3dg_world_get_stats(rp3dg_world* w, rp3dg_world_stats* s) {
    if (!w || !s) return RP3DG_EINVAL;
    *s = w->stats;
    return 0;
}

}  // extern "C"
