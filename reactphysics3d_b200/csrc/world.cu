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
//
// Many worlds step together as a group: each world keeps its own bookkeeping
// (run for all worlds on the host threads, OpenMP) and its own rows of the
// group's device arrays (bodies, colliders, cache slots), while every GPU
// phase is one launch over all worlds: the narrow-phase batches hold the
// pairs of all worlds (algorithm-major), the contact arrays and islands of
// all worlds are packed back to back, and the dynamics stage and collider
// update run on all rows, each world's enabled bodies and colliders given by
// per-row flags.  A single world (rp3dg_world_create) is a group of one.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>


#include <omp.h>

#include "../../include/rp3dg.h"
#include "debug_launch.h"
#include "dynamics_launch.h"
#include "hf_launch.h"
#include "raycast_launch.h"
#include "rp3dg_math.cuh"
#include "world_order.h"

namespace rp3dg {
// (rp3dg_host.cu) host copy of the context's shape table, error message, and
// the dynamics stage / fat-AABB update with per-row enabled flags
int get_shapes_host(rp3dg_ctx* ctx, std::vector<rp3dg_shape>* out);
void set_error(rp3dg_ctx* ctx, const std::string& msg);
int dynamics_step_flags(rp3dg_ctx* ctx, const rp3dg_dynamics_params* pr, const rp3dg_bodies* b,
                        const rp3dg_colliders* c, const rp3dg_manifolds* m, const rp3dg_points* p,
                        const rp3dg_islands* is, const uint8_t* b_enabled, const uint8_t* c_enabled,
                        const DynJoints* joints, const DynTuning* tune, const DynSolver* solver);
int broadphase_update_flags(rp3dg_ctx* ctx, const rp3dg_broadphase* bp, const uint8_t* enabled);
// height fields, the shape table and its local bounds on the device, and the
// triangle tests of convex vs concave pairs
int get_heightfield(rp3dg_ctx* ctx, int32_t id, HfDesc* out);
int get_heightfields(rp3dg_ctx* ctx, std::vector<HfDesc>* out);
int get_mesh_arena_device(rp3dg_ctx* ctx, const uint32_t** words);
int get_mesh_mass(rp3dg_ctx* ctx, int32_t instance, float* volume, float* extent);
int get_mesh_face_counts(rp3dg_ctx* ctx, int32_t instance, std::vector<uint32_t>* counts);
int get_cmeshes(rp3dg_ctx* ctx, std::vector<CmDesc>* out);
int get_shape_device(rp3dg_ctx* ctx, const rp3dg_shape** shapes, const float4** bounds);
int narrowphase_tri_device(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* p, const rp3dg_contact_batch* out,
                           const float4* tri);
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
    const int4* src;            // x item index inside its batch, y batch size, z batch first item, w first point;
                                // concave manifolds: x first point in c_*, y = -1, z points, w first point
    const int4* prev;           // previous pair's manifold start, count, point start, count (x < 0: none)
    const uint8_t* kept_count;  // points kept by the manifold step, per item
    const float4 *b_nd, *b_l1, *b_l2;  // narrow-phase outputs, slot-major per batch (16 slots)
    const float4 *c_nd, *c_l1, *c_l2;  // manifolds of convex vs concave pairs (4 x 4 points per pair)
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
// initContactsWithPreviousOnes (:1069-1160): one thread per manifold; a
// convex pair has one manifold (its narrow-phase slots), a convex vs concave
// pair up to four (from the concave manifold step).
__global__ void __launch_bounds__(128) world_pack_contacts(const PackArgs a) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.nm) return;
    const int4 s = a.src[m];
    const bool concave = s.y < 0;
    const uint32_t k = concave ? uint32_t(s.z) : a.kept_count[uint32_t(s.z + s.x)];
    const uint32_t ps = uint32_t(s.w);
    const uint32_t base = concave ? 0u : uint32_t(s.z) * MAXC;  // batch region start (float4 units)
    a.m_ids[m] = a.ids[m];
    a.m_pstart[m] = ps;
    a.m_npts[m] = uint8_t(k);
    for (uint32_t c = 0; c < k; c++) {
        if (concave) {
            a.p_nd[ps + c] = a.c_nd[uint32_t(s.x) + c];
            a.p_l1[ps + c] = a.c_l1[uint32_t(s.x) + c];
            a.p_l2[ps + c] = a.c_l2[uint32_t(s.x) + c];
        } else {
            const uint32_t src = base + c * uint32_t(s.y) + uint32_t(s.x);
            a.p_nd[ps + c] = a.b_nd[src];
            a.p_l1[ps + c] = a.b_l1[src];
            a.p_l2[ps + c] = a.b_l2[src];
        }
    }
    float4 fv1 = make_float4(0.f, 0.f, 0.f, 0.f), fv2 = fv1, fimp = fv1;
    const int4 pv = a.prev[m];
    if (pv.x >= 0 && k > 0) {
        const float4 cn = concave ? a.c_nd[uint32_t(s.x)] : a.b_nd[base + uint32_t(s.x)];
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
// The velocity condition of the sleep test (updateSleepingBodies,
// PhysicsWorld.cpp:889-893) for every body row: 1 when the squared linear or
// angular speed is above its threshold (the host's float expressions), so
// that the host reads one byte per body instead of both velocities.
__global__ void __launch_bounds__(128) world_sleep_fast(uint32_t n, const float4* __restrict__ lv,
                                                        const float4* __restrict__ av, float slv2, float sav2,
                                                        uint8_t* __restrict__ fast) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 l = lv[i], a = av[i];
    fast[i] = (l.x * l.x + l.y * l.y + l.z * l.z > slv2 || a.x * a.x + a.y * a.y + a.z * a.z > sav2) ? 1 : 0;
}

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

// reportAllShapesOverlappingWithShapes on the GPU: one thread per moved
// collider runs the tree's stack query (same visiting order as
// DynamicAABBTree::reportAllShapesOverlappingWithAABB, DynamicAABBTree.cpp:
// 589-638), counts its leaves, reserves a contiguous block and writes them in
// that order.  A single world with many moved colliders queries a copy of its
// host tree; a world group queries the device trees of its worlds.
constexpr int TREE_STACK = 96;
constexpr size_t TREE_GPU_MIN_QUERIES = 4096;
constexpr size_t DEV_TREE_MAX_COLLIDERS = 8192;   // largest world of a group created with device trees
using TreeNode = rp3dg::order::TreeNode;

__device__ __forceinline__ void tree_query_one(const TreeNode* __restrict__ nodes, int root, int leaf, uint32_t i,
                                               int2* out_pos, int32_t* leaves, uint32_t cap, uint32_t* counter,
                                               uint32_t* flags) {
    const rp3dg::order::Box q = nodes[leaf].box;
    int stack[TREE_STACK];
    auto visit = [&](int32_t* out, uint32_t& cnt) -> bool {
        int sp = 0;
        stack[sp++] = root;
        while (sp > 0) {
            const int id = stack[--sp];
            if (id < 0) continue;
            const rp3dg::order::Box b = nodes[id].box;
            // AABB::testCollision (inclusive)
            if (q.mx[0] < b.mn[0] || b.mx[0] < q.mn[0] || q.mx[1] < b.mn[1] || b.mx[1] < q.mn[1] ||
                q.mx[2] < b.mn[2] || b.mx[2] < q.mn[2])
                continue;
            if (nodes[id].height == 0) {
                if (out) out[cnt] = id;
                cnt++;
            } else {
                if (sp + 2 > TREE_STACK) return false;
                stack[sp++] = nodes[id].child[0];
                stack[sp++] = nodes[id].child[1];
            }
        }
        return true;
    };
    uint32_t cnt = 0;
    if (!visit(nullptr, cnt)) {
        atomicOr(flags, 1u);
        out_pos[i] = make_int2(-1, 0);
        return;
    }
    const uint32_t off = atomicAdd(counter, cnt);
    if (off + cnt > cap) {
        atomicOr(flags, 2u);
        out_pos[i] = make_int2(-1, int(cnt));
        return;
    }
    uint32_t w = 0;
    visit(leaves + off, w);
    out_pos[i] = make_int2(int(off), int(cnt));
}

__global__ void __launch_bounds__(128) world_tree_query(const TreeNode* __restrict__ nodes, int root,
                                                        const int32_t* __restrict__ queries, uint32_t n, int2* out_pos,
                                                        int32_t* leaves, uint32_t cap, uint32_t* counter,
                                                        uint32_t* flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    tree_query_one(nodes, root, queries[i], i, out_pos, leaves, cap, counter, flags);
}

// A world group's trees: world k's nodes are pool[base[k], base[k] + hdr[k].w),
// hdr[k] = (root, first free node, nodes in use, nodes held).  Query i is
// (world, leaf); the moved colliders of a world are consecutive, so the
// threads of a warp mostly walk the same tree.
__global__ void __launch_bounds__(128) world_tree_query_group(const TreeNode* __restrict__ pool,
                                                              const uint32_t* __restrict__ base,
                                                              const int4* __restrict__ hdr,
                                                              const int2* __restrict__ queries, uint32_t n,
                                                              int2* out_pos, int32_t* leaves, uint32_t cap,
                                                              uint32_t* counter, uint32_t* flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 q = queries[i];
    const int4 h = hdr[q.x];
    if (q.y < 0 || q.y >= h.w) {
        atomicOr(flags, 1u);
        out_pos[i] = make_int2(-1, 0);
        return;
    }
    tree_query_one(pool + base[q.x], h.x, q.y, i, out_pos, leaves, cap, counter, flags);
}

// DynamicAABBTree::updateObject's reinsertions (DynamicAABBTree.cpp:186-214,
// removeLeafNode :348-412, insertLeafNode :219-345, balanceSubTreeAtNode
// :420-586) of a world group's moved colliders: one warp per world.  The
// warp reads the world's collider rows 32 at a time (component order, the
// enabled ones first: the order of BroadPhaseSystem::updateCollidersComponents)
// and its first lane replays the reinsertions of the moved ones on the
// world's device tree, in that order.
struct TreeReinsertArgs {
    uint32_t nworlds;
    TreeNode* pool;
    const uint32_t* base;
    int4* hdr;
    const uint2* rows;           // per world: first collider row, colliders
    const uint8_t *enabled, *moved;
    const int32_t* leaf;         // per row: the collider's tree leaf
    const float4 *fmin, *fmax;
    uint32_t* error;             // bit 1: a tree would have had to grow; bit 2: a leaf out of range
};
__global__ void __launch_bounds__(128) world_tree_reinsert(const TreeReinsertArgs a) {
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (k >= a.nworlds) return;
    const uint2 rows = a.rows[k];
    const int4 h = a.hdr[k];
    rp3dg::order::DevTree t;
    t.nodes.p = a.pool + a.base[k];
    t.nodes.n = h.w;
    t.root = h.x;
    t.free_id = h.y;
    t.nb_nodes = h.z;
    bool changed = false, stop = false;
    for (uint32_t r0 = rows.x; r0 < rows.x + rows.y && !stop; r0 += 32) {
        const uint32_t r = r0 + lane;
        const bool in = r < rows.x + rows.y;
        const bool en = in && a.enabled[r];
        const bool mv = en && a.moved[r];
        const unsigned ben = __ballot_sync(0xffffffffu, en);
        unsigned bmv = __ballot_sync(0xffffffffu, mv);
        // the enabled rows come first: the first disabled one ends them
        const unsigned nen = ~ben & ((r0 + 32 <= rows.x + rows.y) ? 0xffffffffu : ((1u << (rows.x + rows.y - r0)) - 1u));
        if (nen) {
            bmv &= (1u << (__ffs(nen) - 1)) - 1u;
            stop = true;
        }
        if (lane == 0) {
            while (bmv) {
                const int b = __ffs(bmv) - 1;
                bmv &= bmv - 1;
                const uint32_t rr = r0 + uint32_t(b);
                const int id = a.leaf[rr];
                if (id < 0 || id >= h.w) {
                    atomicOr(a.error, 2u);
                    stop = true;
                    break;
                }
                const float4 mn = a.fmin[rr], mx = a.fmax[rr];
                rp3dg::order::Box box;
                box.mn[0] = mn.x; box.mn[1] = mn.y; box.mn[2] = mn.z;
                box.mx[0] = mx.x; box.mx[1] = mx.y; box.mx[2] = mx.z;
                t.reinsert(id, box);
                changed = true;
                if (t.failed) {
                    atomicOr(a.error, 1u);
                    stop = true;
                    break;
                }
            }
        }
        stop = __shfl_sync(0xffffffffu, stop, 0);
    }
    if (lane == 0 && changed) a.hdr[k] = make_int4(t.root, t.free_id, t.nb_nodes, t.nodes.n);
}

uint32_t blocks(uint32_t n) { return (n + 127) / 128; }

// ------------------------------------------------------------------ host

// Volume and local inertia tensor of a shape (BoxShape.h:233, BoxShape.cpp:53-59,
// SphereShape.h:170-178, CapsuleShape.h:175-177, CapsuleShape.cpp:51-67).
bool shape_mass(rp3dg_ctx* ctx, const rp3dg_shape& s, float mass_density, float* inertia /*3*/, float* mass_out) {
    const float PI = float(3.141592653589);
    float vol;
    if (s.kind == RP3DG_SHAPE_CONVEX_MESH) {
        // ConvexMeshShape::getVolume and ConvexMesh::getLocalInertiaTensor: the
        // inertia of the box of the scaled bounds
        float ext[3];
        if (rp3dg::get_mesh_mass(ctx, s.mesh, &vol, ext)) return false;
        const float mass = vol * mass_density;
        const float factor = (1.0f / 3.0f) * mass;
        const float xs = ext[0] * ext[0], ys = ext[1] * ext[1], zs = ext[2] * ext[2];
        inertia[0] = factor * (ys + zs);
        inertia[1] = factor * (xs + zs);
        inertia[2] = factor * (xs + ys);
        *mass_out = mass;
        return true;
    }
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
    bool has_sim_collider = false;
    float sleep_time = 0.0f;
    std::vector<int> colliders;
    std::vector<int> joints;       // RigidBodyComponents::mJoints (creation order)
};
struct JointH {
    int type = 0;
    int b1 = -1, b2 = -1;
    bool in_island = false;
    float motor_speed = 0.0f;  // hinge / slider (the record's copy is on the device)
};
struct ColliderH {
    int body = -1;
    int shape = -1;
    bool convex = true;  // CollisionShape::isConvex (height fields and concave meshes are not)
    bool mesh = false;   // a concave collider's shape is a triangle mesh (not a height field)
    int hf = -1;         // height-field or concave-mesh id of a concave collider
    int bp = -1;  // broad-phase id (tree leaf)
    uint16_t category = 1, mask = 0xffff;
    bool trigger = false;  // Collider::setIsTrigger: not a simulation collider
    std::vector<uint64_t> pairs;  // ColliderComponents::mOverlappingPairs
};
struct PairH {
    uint64_t id = 0;
    int bp1 = -1, bp2 = -1;
    int c1 = -1, c2 = -1;  // collider ids
    int algo = 0;
    // OverlappingPair::mNeedToTestOverlap, kept as the world clock's value
    // when it was last cleared: it is set while a collider of the pair has
    // moved since then (need_test below)
    uint64_t reset_at = 0;
    bool coll_prev = false, coll_curr = false, enabled = true;
    int cache = -1;  // slot of its LastFrameCollisionInfo in the device pool
    // convex vs concave pairs (ConcaveOverlappingPair): which shape is convex,
    // and the per-triangle records of the last step that tested the pair
    // (valid only for the step right after it: the others are obsolete)
    bool concave = false, shape1_convex = true, rec_valid = false;
    int rec_start = -1;
    int4 rec_rect = {0, 0, 0, 0};
};
struct ContactPairH {
    uint64_t id;
    int b1, b2, c1, c2;
    uint32_t item;       // global narrow-phase item (convex pair) or concave item
    bool concave = false;
    uint32_t nman = 1;   // manifolds (a convex pair has one)
    uint32_t npts = 0;   // points per manifold, one byte each
    uint32_t k;          // points of all its manifolds after the manifold step
    bool in_island = false;
    bool prev = false;   // ContactPair::collidingInPreviousFrame (the overlapping pair's, at creation)
    bool trigger = false;  // ContactPair::isTrigger: one collider is a trigger (no points, no island)
    uint32_t manifold = 0, point = 0;  // global indices in the packed arrays
};
struct IslandH {
    uint32_t manifold_start = 0, manifold_count = 0;  // world-local manifold range
    uint32_t body_start = 0, body_count = 0;          // its bodies: WorldH::isl_bodies[start, start + count)
};

inline float __int_as_float_host(int v) {
    float f;
    std::memcpy(&f, &v, 4);
    return f;
}

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

// Pair id -> index map for the previous step's contact pairs
// (mPreviousMapPairIdToContactPairIndex): open addressing with linear
// probing over a power-of-two table that is kept from step to step, so
// rebuilding it allocates nothing once it has grown.
struct FlatMap {
    static constexpr uint64_t EMPTY = ~uint64_t(0);
    std::vector<uint64_t> keys;
    std::vector<uint32_t> vals;
    uint32_t mask = 0, n = 0;
    static uint32_t hash(uint64_t k) {
        k ^= k >> 33;
        k *= 0xff51afd7ed558ccdull;
        k ^= k >> 33;
        return uint32_t(k);
    }
    void clear_for(size_t count) {
        size_t cap = 16;
        while (cap < 2 * count) cap <<= 1;
        if (cap != keys.size()) {
            keys.assign(cap, EMPTY);
            vals.assign(cap, 0);
        } else {
            std::fill(keys.begin(), keys.end(), EMPTY);
        }
        mask = uint32_t(cap - 1);
        n = 0;
    }
    void put(uint64_t k, uint32_t v) {
        uint32_t h = hash(k) & mask;
        while (keys[h] != EMPTY && keys[h] != k) h = (h + 1) & mask;
        if (keys[h] == EMPTY) n++;
        keys[h] = k;
        vals[h] = v;
    }
    bool get(uint64_t k, uint32_t& v) const {
        if (keys.empty()) return false;
        uint32_t h = hash(k) & mask;
        while (keys[h] != EMPTY) {
            if (keys[h] == k) {
                v = vals[h];
                return true;
            }
            h = (h + 1) & mask;
        }
        return false;
    }
};

using rp3dg::order::PairMap;


inline uint64_t body_pair_key(int a, int b) {
    return (uint64_t(uint32_t(std::min(a, b))) << 32) | uint32_t(std::max(a, b));
}

// Device columns of the rigid-body components (row = world's first row + component slot).
enum BodyCol { BC_POS, BC_ORI, BC_COMW, BC_COML, BC_LV, BC_AV, BC_F, BC_T, BC_IIL, BC_MASS, BC_LLOCK, BC_ALOCK,
               BC_XC, BC_QC, BC_NCOL };  // XC / QC: constrained position / orientation (joints)
enum ColCol { CC_LPOS, CC_LORI, CC_WPOS, CC_WORI, CC_MAT, CC_FMIN, CC_FMAX, CC_NCOL };

struct ContactBuf {
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

// A tree leaf's collider as the broad phase's candidate filter reads it
// (its body, collision category and mask never change after creation).
struct LeafInfo {
    int32_t body = -1;
    uint16_t category = 0, mask = 0;
};

// One world's order bookkeeping (host) and its rows in the group's arrays.
struct WorldH {
    uint32_t nb = 0, nc = 0, b0 = 0, c0 = 0;  // bodies at rows [b0, b0 + nb), colliders [c0, c0 + nc)
    std::vector<BodyH> bodies;
    std::vector<ColliderH> colliders;
    rp3dg::order::Comps bcomp, ccomp;
    rp3dg::order::Tree tree;
    rp3dg::order::IdSet moved;
    // askForBroadPhaseCollisionCheck marks every pair of a moved collider for
    // the overlap test; instead of visiting them, each mark and each clear
    // takes the next value of this clock (moved_at, PairH::reset_at)
    uint64_t clock = 0;
    std::vector<uint64_t> moved_at;    // by collider id: the clock when it last joined the moved set
    std::vector<int> bp_to_collider;
    std::vector<LeafInfo> leaf_info;   // by tree leaf: what the broad phase's pair filter reads of its collider
    // overlapping pairs (OverlappingPairs::mConvexPairs / mDisabledConvexPairs,
    // mConcavePairs / mDisabledConcavePairs)
    std::vector<PairH> pairs, disabled, concave, concave_dis;
    PairMap map_pairs, map_disabled, map_concave, map_concave_dis;
    std::vector<int> free_cache;
    std::vector<int32_t> reset_slots;
    // contacts of this step and of the previous one
    std::vector<ContactPairH> cpairs, prev_cpairs;
    std::vector<ContactPairH> lost;            // this step's lost contact pairs (mLostContactPairs)
    std::vector<int> isl_bodies;               // the islands' bodies, island after island
    std::vector<uint8_t> sleep_fast;           // the sleep test's velocity condition by body id (reused)
    FlatMap prev_map;
    std::vector<uint32_t> island_order;  // mProcessContactPairsOrderIslands
    std::vector<IslandH> islands;
    std::vector<int> dev_body_at, dev_col_at;  // component order the device rows have
    uint32_t dev_nb_en = ~0u, dev_nc_en = ~0u; // enabled counts the device flags hold
    std::vector<uint8_t> gravity;              // by body id
    // joints: JointComponents and the per-type components (order), the pairs
    // of bodies that must not collide, the first record of this world
    std::vector<JointH> joints;
    rp3dg::order::Comps jcomp, bscomp, fcomp, hcomp, scomp;  // JointComponents, then one per joint type
    PairMap nocollide;   // body pairs (smaller id << 32 | larger id) joined by a joint without collision
    uint32_t jbase = 0;
    struct Pose { float p[3], q[4]; };
    std::vector<Pose> init_pose;               // transforms at creation (joint anchors)
    std::vector<int4> jlist;                   // this step's joints, island by island (record, rows, flags)
    std::vector<uint32_t> isl_jstart, isl_jcount;
    std::vector<int2> jvisit;                  // scratch: (joint, island) in visiting order
    std::vector<int> dfs_stack, dfs_statics;   // scratch of the island search
    std::vector<uint32_t> cp_start, cp_list, cp_fill;   // this step's contact pairs by body (see contacts_and_islands)
    std::vector<uint8_t> b_in_island;          // the island search's marks by body id
    std::vector<int> b_island;                 // this step's island of each non-static body (-1: none)
    std::vector<uint32_t> jfill;               // scratch: next slot of each island's joints
    uint32_t jl_base = 0;
    // islands with joints (group island index), their enabled non-static
    // bodies' rows, and where they go in the group's lists
    std::vector<uint32_t> ji_isl, ji_bcount;
    std::vector<int32_t> ji_rows;
    uint32_t ji_off = 0, ji_row_off = 0;
    bool stepped = false;
    // Body::mIsDebugEnabled by body id, and where the last update's debug
    // primitives of this world start in the group's buffers
    std::vector<uint8_t> body_debug;
    uint32_t dbg_line0 = 0, dbg_nl = 0, dbg_tri0 = 0, dbg_nt = 0;
    // this step
    std::vector<int4> items[NB_ALGOS];
    std::vector<uint32_t> item_pair[NB_ALGOS];
    uint32_t item_off[NB_ALGOS] = {};
    // convex vs concave pairs of the middle phase (hf_launch.h items)
    std::vector<int4> hitems[NB_ALGOS];
    std::vector<uint32_t> hitem_pair[NB_ALGOS];
    uint32_t hitem_off[NB_ALGOS] = {};
    uint32_t nm = 0, np = 0, man_base = 0, pt_base = 0, isl_base = 0;
    double prof_bp[3] = {0.0, 0.0, 0.0};       // broad phase: queries, pair removal, narrow-phase items (ms)
    // tree queries of the moved colliders run on several threads: leaves per
    // thread buffer, and per moved collider (thread, first leaf, count)
    std::vector<std::vector<int>> q_buf;
    std::vector<int4> q_pos;
    std::vector<int32_t> q_shapes;             // this step's moved colliders in the moved set's order
    // one large world's candidate pairs: first candidate of each moved
    // collider, class (0 filtered, 1 existing, 2 new) and existing pair
    std::vector<size_t> c_start;
    std::vector<uint8_t> c_code;
    std::vector<PairH*> c_found;
    uint32_t q_off = 0;                        // their first query in the group's device query list
    // device tree of a world group: whether the host tree's inner nodes are
    // older than the device's (the host keeps the leaves' boxes current)
    bool tree_stale = false;
    std::vector<int> slept;                    // bodies put to sleep by this step
    rp3dg_world_stats stats{};
};

// The per-type joint components (BallAndSocketJointComponents, ...,
// SliderJointComponents) of a joint type.
rp3dg::order::Comps& joint_type_comps(WorldH& w, int type) {
    switch (type) {
        case RP3DG_JOINT_BALL_AND_SOCKET: return w.bscomp;
        case RP3DG_JOINT_FIXED: return w.fcomp;
        case RP3DG_JOINT_HINGE: return w.hcomp;
        default: return w.scomp;
    }
}

}  // namespace

struct rp3dg_world {
    rp3dg_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    rp3dg_world_settings set{};
    std::vector<rp3dg_shape> shapes;
    std::vector<WorldH> worlds;
    uint32_t NB = 0, NC = 0;  // rows of all worlds
    int nthreads = 1;
    std::atomic<uint32_t> cache_next{0};
    // device state
    float4* bcol[2][BC_NCOL] = {};
    float4* biiw[2] = {};
    uint8_t *bgrav = nullptr, *b_en = nullptr, *c_en = nullptr;
    float4* ccol[2][CC_NCOL] = {};
    int32_t *c_body = nullptr, *c_shape = nullptr, *c_leaf = nullptr;   // c_leaf: the collider's tree leaf
    uint16_t *c_cat = nullptr, *c_mask = nullptr;
    uint8_t* c_moved = nullptr;
    int cur_b = 0, cur_c = 0;
    rp3dg_lastframe* pool = nullptr;
    size_t cap_pool = 0;
    int32_t* d_small = nullptr;
    size_t cap_small = 0;
    uint8_t* d_fast = nullptr;     // the sleep test's velocity condition by body row (world_sleep_fast)
    size_t cap_fast = 0;
    bool tables_dirty = true;
    // pinned host copies of the per-row tables and the row permutations
    uint8_t *t_grav = nullptr, *t_ben = nullptr, *t_cen = nullptr;
    int32_t *t_cbody = nullptr, *t_cshape = nullptr, *t_cleaf = nullptr, *t_bperm = nullptr, *t_cperm = nullptr;
    uint16_t *t_cat = nullptr, *t_mask = nullptr;
    // narrow-phase step buffers (all batches of all worlds concatenated)
    size_t cap_items = 0;
    int4* d_items = nullptr;
    int32_t *d_s1 = nullptr, *d_s2 = nullptr;
    float4 *d_p1 = nullptr, *d_r1 = nullptr, *d_p2 = nullptr, *d_r2 = nullptr;
    uint8_t *d_rep = nullptr, *d_coll = nullptr, *d_nct = nullptr;
    rp3dg_lastframe* d_cache = nullptr;
    float4 *d_nd = nullptr, *d_l1 = nullptr, *d_l2 = nullptr;
    uint32_t batch_start[NB_ALGOS + 1] = {};
    // convex vs concave pairs: items (algorithm-major like the batches), their
    // triangle tests, and the per-triangle records of this step and the last
    uint32_t hitem_start[NB_ALGOS + 1] = {};
    uint32_t htest_start[NB_ALGOS + 1] = {};
    rp3dg::HfDesc* d_hf = nullptr;
    uint32_t n_hf = 0;
    rp3dg::CmDesc* d_cm = nullptr;      // concave mesh instances of the context, by id
    uint32_t n_cm = 0;
    int32_t* d_ttri[2] = {nullptr, nullptr};   // per triangle test of a mesh item: its triangle (this step, the last)
    size_t cap_ttri[2] = {0, 0};
    uint32_t *d_herr = nullptr, *h_herr = nullptr;   // middle-phase error word (bit 1: mesh query stack overflow)
    size_t cap_hitem = 0, cap_htest = 0, cap_hc[2] = {0, 0};
    int4 *h_hitems = nullptr, *d_hitems = nullptr, *h_hrect = nullptr, *d_hrect = nullptr;
    uint32_t *h_hstart = nullptr, *d_hstart = nullptr;
    int32_t *h_hpstart = nullptr, *d_hpstart = nullptr;
    int4 *h_hprect = nullptr, *d_hprect = nullptr, *h_hbatch = nullptr, *d_hbatch = nullptr;
    uint8_t *h_hout = nullptr, *d_hout = nullptr;  // points per manifold (4n, uchar4), colliding (n), manifolds (n)
    float4 *d_hond = nullptr, *d_hol1 = nullptr, *d_hol2 = nullptr;
    int32_t *d_ts1 = nullptr, *d_ts2 = nullptr;
    float4 *d_tp1 = nullptr, *d_tr1 = nullptr, *d_tp2 = nullptr, *d_tr2 = nullptr;
    uint8_t *d_trep = nullptr, *d_tcoll = nullptr, *d_tnct = nullptr, *d_tmid = nullptr;
    float4 *d_tnd = nullptr, *d_tl1 = nullptr, *d_tl2 = nullptr, *d_tri = nullptr;
    rp3dg_lastframe* d_tcache[2] = {nullptr, nullptr};
    int cur_tc = 0;
    cudaEvent_t ev_rect = nullptr;
    // island scheduling and its autotuner: candidates are tried on successive
    // steps (round robin, `rounds` times each), timed with CUDA events around
    // the dynamics stage per manifold, one parameter after the other
    rp3dg::DynTuning tune{};
    struct Tuner {
        bool active = false;
        int phase = 0, rounds = 2, idx = 0;
        std::vector<rp3dg::DynTuning> cands;
        std::vector<std::vector<float>> score;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        bool timed = false;
        uint32_t nm = 0;
    } tuner;
    // broad-phase tree queries on the GPU (worlds with many moved colliders)
    TreeNode *h_tnodes = nullptr, *d_tnodes = nullptr;
    size_t cap_tnodes = 0, cap_tq = 0, cap_tleaves = 0, cap_tpos = 0, cap_tcnt = 0;
    int32_t *h_tq = nullptr, *d_tq = nullptr, *h_tleaves = nullptr, *d_tleaves = nullptr;
    int2 *h_tpos = nullptr, *d_tpos = nullptr;
    uint32_t *h_tcnt = nullptr, *d_tcnt = nullptr;   // [0] leaves reserved, [1] flags, [2] reinsertion errors
    // world groups: every world's broad-phase tree in one device pool (world
    // k's nodes from tree_base[k], header root / free node / nodes in use /
    // nodes held), reinserted and queried on the GPU; the host replica keeps the
    // moved set, the leaves' boxes and the pairs
    bool dev_tree = false;
    TreeNode* d_tree = nullptr;
    uint32_t* d_tree_base = nullptr;
    int4* d_tree_hdr = nullptr;
    uint2* d_tree_rows = nullptr;                    // per world: first collider row, colliders
    std::vector<uint32_t> tree_base;
    size_t cap_gq = 0;
    int2 *h_gq = nullptr, *d_gq = nullptr;           // queries (world, leaf)
    cudaEvent_t ev_step_copy = nullptr;              // the step's moved flags and fat AABBs are on the host
    // world raycasts: the tree's nodes and the collider table as the ray
    // kernel reads them (rebuilt when the world state changed), rays and hits
    uint64_t state_version = 1;      // bumped by every update and between-step change
    uint64_t ray_version = 0;        // state the ray tables were built for
    uint32_t ray_world = 0;
    rp3dg::RayNode *h_rnodes = nullptr, *d_rnodes = nullptr;
    int4 *h_rcols = nullptr, *d_rcols = nullptr;
    size_t cap_rnodes = 0, cap_rcols = 0, cap_rhf = 0, cap_rays = 0, cap_rhits = 0, cap_rcount = 0;
    rp3dg::HfDesc* d_rhf = nullptr;
    uint32_t nb_rhf = 0;
    rp3dg_ray* d_rays = nullptr;
    rp3dg_raycast_hit* d_rhits = nullptr;
    uint32_t* d_rcount = nullptr;    // n counts, then the error word
    cudaEvent_t ev_r0 = nullptr, ev_r1 = nullptr;
    // manifold packing
    size_t cap_m = 0, cap_i = 0;
    int4 *d_mids = nullptr, *d_msrc = nullptr, *d_mprev = nullptr;
    uint32_t *d_istart = nullptr, *d_icount = nullptr;
    ContactBuf cbuf[2];
    int cur_cb = 0;
    // joints: records by global joint index, per-step lists
    rp3dg::JointRec* j_rec = nullptr;
    uint32_t nj_total = 0;
    size_t cap_jrec = 0;
    int4* d_jlist = nullptr;
    uint32_t *d_ijstart = nullptr, *d_ijcount = nullptr, *d_jiisl = nullptr, *d_jibstart = nullptr, *d_jibcount = nullptr;
    int32_t* d_jirows = nullptr;
    size_t cap_jl = 0, cap_ji = 0, cap_jbs = 0, cap_jbc = 0, cap_jr = 0;
    // pinned host staging
    size_t cap_hitems = 0, cap_hout = 0, cap_hm = 0, cap_hi = 0, cap_hstep = 0, cap_hreset = 0;
    int4* h_items = nullptr;
    uint8_t* h_out = nullptr;  // colliding flag, kept count
    int4 *h_mids = nullptr, *h_msrc = nullptr, *h_mprev = nullptr;
    uint32_t *h_istart = nullptr, *h_icount = nullptr, *h_ijstart = nullptr, *h_ijcount = nullptr;
    int4* h_jlist = nullptr;
    size_t cap_hjl = 0;
    uint8_t* h_step = nullptr;  // moved flags, fat AABBs, velocities after the step
    int32_t* h_reset = nullptr;
    // solver (rp3dg_world_set_solver): 0 exact order, 1 graph-coloured;
    // with stats, each step's solver statistics in d_solver_stats
    int solver = 0;
    bool solver_stats = false;
    rp3dg::SolverStats* d_solver_stats = nullptr;
    // debug rendering (rp3dg_world_set_debug_rendering): the items shown,
    // the collider transforms before the integration of the last update
    // (world positions then orientations, NC rows each) and that update's
    // primitives, world after world
    uint32_t debug_items = 0;
    float4* d_dbg_snap = nullptr;
    rp3dg_debug_line* d_dbg_lines = nullptr;
    rp3dg_debug_triangle* d_dbg_tris = nullptr;
    rp3dg::DebugJob* d_dbg_jobs = nullptr;
    int4* d_dbg_points = nullptr;
    size_t cap_dbg_snap = 0, cap_dbg_lines = 0, cap_dbg_tris = 0, cap_dbg_jobs = 0, cap_dbg_points = 0;
    // phase profiling (rp3dg_world_set_profiling): cumulative ms per phase
    bool profiling = false;
    double phase_ms[16] = {};
    std::chrono::steady_clock::time_point t_mark;
    rp3dg_world_stats stats{};
};

namespace {

using Group = rp3dg_world;

int wfail(Group* g, int code, const std::string& msg) {
    if (g) rp3dg::set_error(g->ctx, "world: " + msg);
    return code;
}
int cfail(rp3dg_ctx* ctx, int code, const std::string& msg) {
    rp3dg::set_error(ctx, "world: " + msg);
    return code;
}
int wcuda(Group* g, cudaError_t e, const char* what) {
    return wfail(g, RP3DG_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
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

// Cache slots: a world takes chunks of the group's pool and keeps a free list.
int alloc_cache(Group* g, WorldH& w) {
    if (w.free_cache.empty()) {
        constexpr uint32_t CHUNK = 64;
        const uint32_t base = g->cache_next.fetch_add(CHUNK);
        for (uint32_t i = CHUNK; i-- > 0;) w.free_cache.push_back(int(base + i));
    }
    const int slot = w.free_cache.back();
    w.free_cache.pop_back();
    w.reset_slots.push_back(slot);
    return slot;
}

// OverlappingPairs::getOverlappingPair
PairH* find_pair(WorldH& w, uint64_t id) {
    auto it = w.map_pairs.find(id);
    if (it != w.map_pairs.end()) return &w.pairs[it->second];
    it = w.map_concave.find(id);
    if (it != w.map_concave.end()) return &w.concave[it->second];
    it = w.map_disabled.find(id);
    if (it != w.map_disabled.end()) return &w.disabled[it->second];
    it = w.map_concave_dis.find(id);
    if (it != w.map_concave_dis.end()) return &w.concave_dis[it->second];
    return nullptr;
}

// swap-remove from a pair array keeping its id map (removeConvexPairWithIndex)
void remove_pair_at(std::vector<PairH>& arr, PairMap& map, uint32_t idx) {
    map.erase(arr[idx].id);
    const uint32_t last = uint32_t(arr.size()) - 1;
    if (arr.size() > 1 && idx < last) map[arr[last].id] = idx;
    arr[idx] = arr[last];
    arr.pop_back();
}

void remove_from_collider(WorldH& w, int c, uint64_t id) {
    auto& v = w.colliders[size_t(c)].pairs;
    auto it = std::find(v.begin(), v.end(), id);
    if (it != v.end()) v.erase(it);
}

// OverlappingPairs::addPair (OverlappingPairs.cpp:397-449): a convex pair, or
// a convex vs concave pair whose algorithm is the convex shape's against a
// CONVEX_POLYHEDRON (the triangles)
void add_pair(Group* g, WorldH& w, int c1, int c2) {
    const ColliderH &C1 = w.colliders[size_t(c1)], &C2 = w.colliders[size_t(c2)];
    const uint32_t b1 = uint32_t(C1.bp), b2 = uint32_t(C2.bp);
    PairH p;
    p.id = pair_number(std::max(b1, b2), std::min(b1, b2));
    p.reset_at = ++w.clock;
    p.bp1 = int(b1);
    p.bp2 = int(b2);
    p.c1 = c1;
    p.c2 = c2;
    p.enabled = true;
    if (C1.convex && C2.convex) {
        p.algo = select_algorithm(shape_type_index(g->shapes[size_t(C1.shape)]),
                                  shape_type_index(g->shapes[size_t(C2.shape)]));
        p.cache = alloc_cache(g, w);
        w.map_pairs[p.id] = uint32_t(w.pairs.size());
        w.pairs.push_back(p);
    } else {
        p.concave = true;
        p.shape1_convex = C1.convex;
        p.algo = select_algorithm(shape_type_index(g->shapes[size_t(C1.convex ? C1.shape : C2.shape)]), 2);
        w.map_concave[p.id] = uint32_t(w.concave.size());
        w.concave.push_back(p);
    }
    w.colliders[size_t(c1)].pairs.push_back(p.id);
    w.colliders[size_t(c2)].pairs.push_back(p.id);
}

// CollisionDetectionSystem::addLostContactPair (CollisionDetectionSystem.cpp:220-236)
void add_lost(WorldH& w, const PairH& p) {
    ContactPairH c;
    c.id = p.id;
    c.c1 = p.c1;
    c.c2 = p.c2;
    c.b1 = w.colliders[size_t(p.c1)].body;
    c.b2 = w.colliders[size_t(p.c2)].body;
    c.prev = true;
    c.k = 0;
    c.trigger = w.colliders[size_t(p.c1)].trigger || w.colliders[size_t(p.c2)].trigger;
    w.lost.push_back(c);
}

// removeConvexPairWithIndex(index, removeFromColliders = true)
void remove_pair(WorldH& w, uint32_t idx) {
    PairH& p = w.pairs[idx];
    remove_from_collider(w, p.c1, p.id);
    remove_from_collider(w, p.c2, p.id);
    w.free_cache.push_back(p.cache);
    remove_pair_at(w.pairs, w.map_pairs, idx);
}

// removeConcavePairWithIndex(index, removeFromColliders = true): its
// per-triangle records go with it
void remove_concave_pair(WorldH& w, uint32_t idx) {
    PairH& p = w.concave[idx];
    remove_from_collider(w, p.c1, p.id);
    remove_from_collider(w, p.c2, p.id);
    remove_pair_at(w.concave, w.map_concave, idx);
}

// disableConvexPairWithIndex / enableConvexPairWithIndex: the pair is
// re-created in the other array with a fresh temporal-coherence record
void disable_pair(Group* g, WorldH& w, uint64_t id) {
    auto it = w.map_pairs.find(id);
    if (it == w.map_pairs.end()) {
        // disableConcavePairWithIndex: re-created without records
        auto ic = w.map_concave.find(id);
        if (ic == w.map_concave.end()) return;
        const uint32_t idx = ic->second;
        PairH np = w.concave[idx];
        np.enabled = false;
        np.reset_at = ++w.clock;
        np.rec_valid = false;
        w.map_concave_dis[id] = uint32_t(w.concave_dis.size());
        w.concave_dis.push_back(np);
        remove_pair_at(w.concave, w.map_concave, idx);
        return;
    }
    const uint32_t idx = it->second;
    PairH np = w.pairs[idx];
    np.enabled = false;
    np.reset_at = ++w.clock;
    w.free_cache.push_back(np.cache);
    np.cache = alloc_cache(g, w);
    w.map_disabled[id] = uint32_t(w.disabled.size());
    w.disabled.push_back(np);
    remove_pair_at(w.pairs, w.map_pairs, idx);
}
void enable_pair(Group* g, WorldH& w, uint64_t id) {
    auto it = w.map_disabled.find(id);
    if (it == w.map_disabled.end()) {
        // enableConcavePairWithIndex
        auto ic = w.map_concave_dis.find(id);
        if (ic == w.map_concave_dis.end()) return;
        const uint32_t idx = ic->second;
        PairH np = w.concave_dis[idx];
        np.enabled = true;
        np.reset_at = ++w.clock;
        np.rec_valid = false;
        w.map_concave[id] = uint32_t(w.concave.size());
        w.concave.push_back(np);
        remove_pair_at(w.concave_dis, w.map_concave_dis, idx);
        return;
    }
    const uint32_t idx = it->second;
    PairH np = w.disabled[idx];
    np.enabled = true;
    np.reset_at = ++w.clock;
    w.free_cache.push_back(np.cache);
    np.cache = alloc_cache(g, w);
    w.map_pairs[id] = uint32_t(w.pairs.size());
    w.pairs.push_back(np);
    remove_pair_at(w.disabled, w.map_disabled, idx);
}

// BroadPhaseSystem::addMovedCollider + notifyOverlappingPairsToTestOverlap
void add_moved(WorldH& w, int c) {
    w.moved.add(w.colliders[size_t(c)].bp);
    w.moved_at[size_t(c)] = ++w.clock;
}

// OverlappingPair::needToTestOverlap
bool need_test(const WorldH& w, const PairH& p) {
    return w.moved_at[size_t(p.c1)] > p.reset_at || w.moved_at[size_t(p.c2)] > p.reset_at;
}

// PhysicsWorld::setBodyDisabled (PhysicsWorld.cpp:168-186)
void set_body_disabled(WorldH& w, int b, bool dis) {
    if (w.bcomp.enabled(b) == !dis) return;
    w.bcomp.set_disabled(b, dis);
    for (int c : w.bodies[size_t(b)].colliders) w.ccomp.set_disabled(c, dis);
}

// RigidBody::setIsSleeping (RigidBody.cpp:1006-1057)
void set_sleeping(Group* g, WorldH& w, int b, bool sleeping) {
    BodyH& B = w.bodies[size_t(b)];
    if (B.sleeping == sleeping) return;
    if (B.type == RP3DG_BODY_STATIC) return;
    if (sleeping) B.sleep_time = 0.0f;
    else if (B.sleeping) B.sleep_time = 0.0f;
    B.sleeping = sleeping;
    set_body_disabled(w, b, sleeping);
    if (sleeping) {
        // checkForDisabledOverlappingPairs
        for (int c : B.colliders) {
            const std::vector<uint64_t> ids = w.colliders[size_t(c)].pairs;
            for (uint64_t id : ids) {
                PairH* p = find_pair(w, id);
                if (!p) continue;
                const int o1 = w.colliders[size_t(p->c1)].body, o2 = w.colliders[size_t(p->c2)].body;
                if (!w.bcomp.enabled(o1) && !w.bcomp.enabled(o2)) disable_pair(g, w, id);
            }
        }
        w.slept.push_back(b);
    } else {
        // enableOverlappingPairs + askForBroadPhaseCollisionCheck
        for (int c : B.colliders) {
            const std::vector<uint64_t> ids = w.colliders[size_t(c)].pairs;
            for (uint64_t id : ids) {
                PairH* p = find_pair(w, id);
                if (p && !p->enabled) enable_pair(g, w, id);
            }
        }
        for (int c : B.colliders) add_moved(w, c);
    }
}

// ---------------------------------------------------------------- phases

// Pinned host and device copies of one array, grown together.
template <class T>
bool pair_grow(T** h, T** d, size_t* cap, size_t need) {
    if (need <= *cap && *h && *d) return true;
    const size_t n = std::max<size_t>(std::max<size_t>(need, *cap * 2), 256);
    cudaFreeHost(*h);
    cudaFree(*d);
    *h = nullptr;
    *d = nullptr;
    *cap = 0;
    if (cudaMallocHost(reinterpret_cast<void**>(h), n * sizeof(T)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(d), n * sizeof(T)) != cudaSuccess)
        return false;
    *cap = n;
    return true;
}

// The moved colliders' tree queries on the GPU: the leaves of query i are
// h_tleaves[pos.x, pos.x + pos.y) (pos = h_tpos[i]) in the host query's
// order.  False when a buffer cannot be had or a query needs a deeper stack
// (the caller then queries on the host).
bool tree_queries_gpu(Group* g, WorldH& w, const std::vector<int32_t>& shapes) {
    const size_t nn = w.tree.nodes.size(), nq = shapes.size();
    cudaStream_t st = g->stream;
    if (!pair_grow(&g->h_tnodes, &g->d_tnodes, &g->cap_tnodes, nn) || !pair_grow(&g->h_tq, &g->d_tq, &g->cap_tq, nq) ||
        !pair_grow(&g->h_tpos, &g->d_tpos, &g->cap_tpos, nq) ||
        !pair_grow(&g->h_tcnt, &g->d_tcnt, &g->cap_tcnt, 2) ||
        !pair_grow(&g->h_tleaves, &g->d_tleaves, &g->cap_tleaves, 8 * nq))
        return false;
    std::memcpy(g->h_tnodes, w.tree.nodes.data(), nn * sizeof(TreeNode));
    std::memcpy(g->h_tq, shapes.data(), nq * 4);
    cudaMemcpyAsync(g->d_tnodes, g->h_tnodes, nn * sizeof(TreeNode), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(g->d_tq, g->h_tq, nq * 4, cudaMemcpyHostToDevice, st);
    for (int attempt = 0; attempt < 2; attempt++) {
        cudaMemsetAsync(g->d_tcnt, 0, 8, st);
        world_tree_query<<<blocks(uint32_t(nq)), 128, 0, st>>>(g->d_tnodes, w.tree.root, g->d_tq, uint32_t(nq),
                                                               g->d_tpos, g->d_tleaves, uint32_t(g->cap_tleaves),
                                                               g->d_tcnt, g->d_tcnt + 1);
        cudaMemcpyAsync(g->h_tcnt, g->d_tcnt, 8, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return false;
        const uint32_t total = g->h_tcnt[0], flags = g->h_tcnt[1];
        if (flags & 1u) return false;
        if (flags & 2u) {
            if (attempt || !pair_grow(&g->h_tleaves, &g->d_tleaves, &g->cap_tleaves, size_t(total) + 1024)) return false;
            continue;
        }
        cudaMemcpyAsync(g->h_tpos, g->d_tpos, nq * sizeof(int2), cudaMemcpyDeviceToHost, st);
        if (total) cudaMemcpyAsync(g->h_tleaves, g->d_tleaves, size_t(total) * 4, cudaMemcpyDeviceToHost, st);
        return cudaStreamSynchronize(st) == cudaSuccess;
    }
    return false;
}

// computeBroadPhase (CollisionDetectionSystem.cpp:103-167, 270-343) and the
// middle phase for convex pairs (:346-410): narrow-phase items in pair order.
void broad_and_middle_phase(Group* g, WorldH& w) {
    using clk = std::chrono::steady_clock;
    const auto t0 = g->profiling ? clk::now() : clk::time_point();
    // with device trees the group's queries ran before (tree_queries_group)
    const bool dev = g->dev_tree;
    std::vector<int32_t>& shapes = w.q_shapes;
    if (!dev) {
        w.moved.to_array(shapes);
        w.moved.clear();
    }
    // reportAllShapesOverlappingWithShapes: the tree does not change during
    // the queries, so with a single world on the group's threads they run in
    // parallel; the pairs are then processed in the moved set's order
    const int nt = (!dev && g->nthreads > 1 && g->worlds.size() == 1 && shapes.size() >= 256) ? g->nthreads : 1;
    // a single world with many moved colliders queries on the GPU
    const bool gpu = dev || (g->worlds.size() == 1 && shapes.size() >= TREE_GPU_MIN_QUERIES &&
                             tree_queries_gpu(g, w, shapes));
    const uint32_t qbase = dev ? w.q_off : 0;
    if (int(w.q_buf.size()) < nt) w.q_buf.resize(size_t(nt));
    w.q_pos.resize(shapes.size());
#pragma omp parallel num_threads(nt) if (nt > 1 && !gpu)
    if (!gpu) {
        const int t = omp_get_thread_num();
        std::vector<int>& buf = w.q_buf[size_t(t)];
        buf.clear();
        std::vector<int> stack;
#pragma omp for schedule(static)
        for (long i = 0; i < long(shapes.size()); i++) {
            const size_t o = buf.size();
            w.tree.query(w.tree.nodes[size_t(shapes[size_t(i)])].box, buf, stack);
            w.q_pos[size_t(i)] = make_int4(t, int(o), int(buf.size() - o), 0);
        }
    }
    auto leaves_of = [&](size_t i, const int** leaves, int* nleaf) {
        if (gpu) {
            const int2 tp = g->h_tpos[qbase + i];
            *leaves = g->h_tleaves + tp.x;
            *nleaf = tp.y;
        } else {
            const int4 qp = w.q_pos[i];
            *leaves = w.q_buf[size_t(qp.x)].data() + qp.y;
            *nleaf = qp.z;
        }
    };
    // a candidate pair of the queries: 0 filtered out, 1 an existing pair, 2 new
    auto classify = [&](int32_t s, int leaf, PairH** found) -> uint8_t {
        if (leaf == s) return 0;
        const LeafInfo &L1 = w.leaf_info[size_t(s)], &L2 = w.leaf_info[size_t(leaf)];
        if (L1.body == L2.body) return 0;
        if (!w.nocollide.empty() && w.nocollide.find(body_pair_key(L1.body, L2.body))) return 0;
        *found = find_pair(w, pair_number(uint32_t(std::max(s, leaf)), uint32_t(std::min(s, leaf))));
        return *found ? 1 : 2;
    };
    auto add_new = [&](int32_t s, int leaf) {
        const uint64_t id = pair_number(uint32_t(std::max(s, leaf)), uint32_t(std::min(s, leaf)));
        PairH* p = find_pair(w, id);
        if (p) {
            p->reset_at = ++w.clock;
            return;
        }
        const int c1 = w.bp_to_collider[size_t(s)], c2 = w.bp_to_collider[size_t(leaf)];
        const ColliderH &C1 = w.colliders[size_t(c1)], &C2 = w.colliders[size_t(c2)];
        if ((C1.mask & C2.category) != 0 && (C1.category & C2.mask) != 0 && (C1.convex || C2.convex))
            add_pair(g, w, c1, c2);
    };
    if (g->worlds.size() == 1 && g->nthreads > 1 && shapes.size() >= 256) {
        // one large world: the candidates are classified on the group's
        // threads (lookups only), the existing pairs' marks cleared (all
        // with one clock value: every mark this clears is older), and only
        // the new ones are added in the moved set's order, each looked up
        // again so that a pair met twice is added once
        size_t total = 0;
        w.c_start.resize(shapes.size() + 1);
        for (size_t i = 0; i < shapes.size(); i++) {
            const int* lv;
            int nl;
            leaves_of(i, &lv, &nl);
            w.c_start[i] = total;
            total += size_t(nl);
        }
        w.c_start[shapes.size()] = total;
        w.c_code.resize(total);
        w.c_found.resize(total);
#pragma omp parallel for schedule(dynamic, 64) num_threads(g->nthreads)
        for (long i = 0; i < long(shapes.size()); i++) {
            const int* lv;
            int nl;
            leaves_of(size_t(i), &lv, &nl);
            const size_t o = w.c_start[size_t(i)];
            for (int li = 0; li < nl; li++) {
                PairH* f = nullptr;
                w.c_code[o + size_t(li)] = classify(shapes[size_t(i)], lv[li], &f);
                w.c_found[o + size_t(li)] = f;
            }
        }
        const uint64_t stamp = ++w.clock;
        for (size_t j = 0; j < total; j++)
            if (w.c_code[j] == 1) w.c_found[j]->reset_at = stamp;
        for (size_t i = 0; i < shapes.size(); i++) {
            const int* lv;
            int nl;
            leaves_of(i, &lv, &nl);
            const size_t o = w.c_start[i];
            for (int li = 0; li < nl; li++)
                if (w.c_code[o + size_t(li)] == 2) add_new(shapes[i], lv[li]);
        }
    } else {
        for (size_t i = 0; i < shapes.size(); i++) {
            const int* lv;
            int nl;
            leaves_of(i, &lv, &nl);
            for (int li = 0; li < nl; li++) {
                PairH* f = nullptr;
                const uint8_t code = classify(shapes[i], lv[li], &f);
                if (code == 1) f->reset_at = ++w.clock;
                else if (code == 2) add_new(shapes[i], lv[li]);
            }
        }
    }
    const auto t1 = g->profiling ? clk::now() : clk::time_point();
    // removeNonOverlappingPairs; a pair removed while it was colliding in
    // the previous frame becomes a lost contact pair (addLostContactPair)
    // (collidingInPreviousFrame is the last step's coll_curr here: it moves
    // into coll_prev in the item loops below)
    w.lost.clear();
    for (uint64_t i = 0; i < w.pairs.size(); i++) {
        PairH& p = w.pairs[i];
        if (!need_test(w, p)) continue;
        if (rp3dg::order::overlap(w.tree.nodes[size_t(p.bp1)].box, w.tree.nodes[size_t(p.bp2)].box)) {
            p.reset_at = ++w.clock;
        } else {
            if (p.coll_curr) add_lost(w, p);
            remove_pair(w, uint32_t(i));
            i--;
        }
    }
    for (uint64_t i = 0; i < w.concave.size(); i++) {
        PairH& p = w.concave[i];
        if (!need_test(w, p)) continue;
        if (rp3dg::order::overlap(w.tree.nodes[size_t(p.bp1)].box, w.tree.nodes[size_t(p.bp2)].box)) {
            p.reset_at = ++w.clock;
        } else {
            if (p.coll_curr) add_lost(w, p);
            remove_concave_pair(w, uint32_t(i));
            i--;
        }
    }
    const auto t2 = g->profiling ? clk::now() : clk::time_point();
    for (int a = 0; a < NB_ALGOS; a++) {
        w.items[a].clear();
        w.item_pair[a].clear();
        w.hitems[a].clear();
        w.hitem_pair[a].clear();
    }
    // rows in the order the device will have after this step's row sync;
    // each pair's collidingInPreviousFrame is its last step's flag (for the
    // enabled pairs, which are the ones the reference updates at the end of
    // a step; a disabled pair keeps both flags as they were)
    for (uint32_t i = 0; i < w.pairs.size(); i++) {
        PairH& p = w.pairs[i];
        p.coll_prev = p.coll_curr;
        p.coll_curr = false;
        const bool e1 = w.ccomp.enabled(p.c1), e2 = w.ccomp.enabled(p.c2);
        if (!(e1 || e2)) continue;
        const int a = p.algo - 1;
        // reportContacts is off when a collider is a trigger (:402)
        const bool trig = w.colliders[size_t(p.c1)].trigger || w.colliders[size_t(p.c2)].trigger;
        w.items[a].push_back(make_int4(int(w.c0) + w.ccomp.slot[size_t(p.c1)], int(w.c0) + w.ccomp.slot[size_t(p.c2)],
                                       p.cache, trig ? 0 : 1));
        w.item_pair[a].push_back(i);
    }
    // convex vs concave pairs (computeMiddlePhase :412-456): a pair that is
    // not tested this step loses its per-triangle records
    for (uint32_t i = 0; i < w.concave.size(); i++) {
        PairH& p = w.concave[i];
        p.coll_prev = p.coll_curr;
        p.coll_curr = false;
        const bool e1 = w.ccomp.enabled(p.c1), e2 = w.ccomp.enabled(p.c2);
        if (!(e1 || e2)) {
            p.rec_valid = false;
            continue;
        }
        const int cv = p.shape1_convex ? p.c1 : p.c2, cc = p.shape1_convex ? p.c2 : p.c1;
        const int a = p.algo - 1;
        const bool trig = w.colliders[size_t(p.c1)].trigger || w.colliders[size_t(p.c2)].trigger;
        w.hitems[a].push_back(make_int4(int(w.c0) + w.ccomp.slot[size_t(cv)], int(w.c0) + w.ccomp.slot[size_t(cc)],
                                        w.colliders[size_t(cc)].hf,
                                        (p.shape1_convex ? HF_SHAPE1_CONVEX : 0) | (trig ? HF_NO_REPORT : 0) |
                                            (w.colliders[size_t(cc)].mesh ? HF_MESH : 0)));
        w.hitem_pair[a].push_back(i);
    }
    if (g->profiling) {
        const auto t3 = clk::now();
        w.prof_bp[0] += std::chrono::duration<double, std::milli>(t1 - t0).count();
        w.prof_bp[1] += std::chrono::duration<double, std::milli>(t2 - t1).count();
        w.prof_bp[2] += std::chrono::duration<double, std::milli>(t3 - t2).count();
    }
}

// processAllPotentialContacts' contact pairs (batch order), addContactPairsToBodies
// and PhysicsWorld::createIslands (PhysicsWorld.cpp:695-866).
void contacts_and_islands(Group* g, WorldH& w, const uint8_t* h_coll, const uint8_t* h_count, const uint8_t* h_hcoll,
                          const uint8_t* h_hnman, const uint8_t* h_hnpts) {
    w.cpairs.clear();
    // batch by batch; inside a batch the convex pairs' tests come first, then
    // the triangles of the concave pairs (computeMiddlePhase's order)
    for (int a = 0; a < NB_ALGOS; a++) {
        const uint32_t base = g->batch_start[a] + w.item_off[a];
        for (uint32_t i = 0; i < w.items[a].size(); i++) {
            const uint32_t it = base + i;
            if (!h_coll[it]) continue;
            PairH& p = w.pairs[w.item_pair[a][i]];
            p.coll_curr = true;
            ContactPairH c;
            c.prev = p.coll_prev;
            c.id = p.id;
            c.c1 = p.c1;
            c.c2 = p.c2;
            c.b1 = w.colliders[size_t(p.c1)].body;
            c.b2 = w.colliders[size_t(p.c2)].body;
            c.item = it;
            c.k = h_count[it];
            c.npts = c.k;
            c.trigger = w.colliders[size_t(p.c1)].trigger || w.colliders[size_t(p.c2)].trigger;
            if (c.trigger) c.nman = 0;   // a trigger pair has no contact points, so no manifold
            w.cpairs.push_back(c);
        }
        const uint32_t hbase = g->hitem_start[a] + w.hitem_off[a];
        for (uint32_t i = 0; i < w.hitems[a].size(); i++) {
            const uint32_t it = hbase + i;
            if (!h_hcoll[it]) continue;
            PairH& p = w.concave[w.hitem_pair[a][i]];
            p.coll_curr = true;
            ContactPairH c;
            c.prev = p.coll_prev;
            c.id = p.id;
            c.c1 = p.c1;
            c.c2 = p.c2;
            c.b1 = w.colliders[size_t(p.c1)].body;
            c.b2 = w.colliders[size_t(p.c2)].body;
            c.item = it;
            c.concave = true;
            c.trigger = w.colliders[size_t(p.c1)].trigger || w.colliders[size_t(p.c2)].trigger;
            c.nman = c.trigger ? 0u : h_hnman[it];
            c.k = 0;
            c.npts = 0;
            for (uint32_t m = 0; m < c.nman; m++) {
                c.k += h_hnpts[4 * size_t(it) + m];
                c.npts |= uint32_t(h_hnpts[4 * size_t(it) + m]) << (8 * m);
            }
            w.cpairs.push_back(c);
        }
    }
    // computeLostContactPairs (CollisionDetectionSystem.cpp:978-1011): pairs
    // colliding in the previous frame and not in this one, convex then concave
    for (const PairH& p : w.pairs)
        if (p.coll_prev && !p.coll_curr) add_lost(w, p);
    for (const PairH& p : w.concave)
        if (p.coll_prev && !p.coll_curr) add_lost(w, p);
    // each body's contact pairs in creation order (RigidBodyComponents'
    // contact pair lists), as one array per world: body b's are
    // cp_list[cp_start[b], cp_start[b + 1])
    {
        std::vector<uint32_t>& cs = w.cp_start;
        cs.assign(w.bodies.size() + 1, 0);
        for (const ContactPairH& c : w.cpairs) {
            cs[size_t(c.b1) + 1]++;
            cs[size_t(c.b2) + 1]++;
        }
        for (size_t b = 0; b < w.bodies.size(); b++) cs[b + 1] += cs[b];
        w.cp_list.resize(2 * w.cpairs.size());
        std::vector<uint32_t>& fill = w.cp_fill;
        fill.assign(cs.begin(), cs.end() - 1);
        for (uint32_t p = 0; p < w.cpairs.size(); p++) {
            w.cp_list[fill[size_t(w.cpairs[p].b1)]++] = p;
            w.cp_list[fill[size_t(w.cpairs[p].b2)]++] = p;
        }
    }
    w.island_order.clear();
    w.islands.clear();
    w.isl_bodies.clear();
    // the search's per-body marks, in arrays of their own (cheaper to reset
    // and to test than the body records)
    std::vector<uint8_t>& in_island = w.b_in_island;
    std::vector<int>& island_of = w.b_island;
    in_island.assign(w.bodies.size(), 0);
    island_of.assign(w.bodies.size(), -1);
    for (auto& J : w.joints) J.in_island = false;
    uint32_t total_manifolds = 0;
    std::vector<int>& stack = w.dfs_stack;
    std::vector<int>& statics = w.dfs_statics;
    statics.clear();
    for (uint32_t s = 0; s < w.bcomp.n_enabled; s++) {
        const int b0 = w.bcomp.at[s];
        if (in_island[size_t(b0)]) continue;
        if (w.bodies[size_t(b0)].type == RP3DG_BODY_STATIC) continue;
        stack.clear();
        in_island[size_t(b0)] = true;
        stack.push_back(b0);
        IslandH isl;
        isl.manifold_start = total_manifolds;
        isl.body_start = uint32_t(w.isl_bodies.size());
        const size_t isl_index = w.islands.size();
        w.islands.push_back(isl);
        while (!stack.empty()) {
            const int b = stack.back();
            stack.pop_back();
            w.isl_bodies.push_back(b);
            w.islands[isl_index].body_count++;
            set_sleeping(g, w, b, false);
            if (w.bodies[size_t(b)].type == RP3DG_BODY_STATIC) {
                statics.push_back(b);
                continue;
            }
            island_of[size_t(b)] = int(isl_index);
            for (uint32_t k = w.cp_start[size_t(b)]; k < w.cp_start[size_t(b) + 1]; k++) {
                const uint32_t cpi = w.cp_list[k];
                ContactPairH& cp = w.cpairs[cpi];
                if (cp.in_island) continue;
                cp.in_island = true;
                // both colliders must be simulation colliders (:788-790)
                if (cp.trigger) continue;
                const int other = cp.b1 == b ? cp.b2 : cp.b1;
                if (w.bodies[size_t(other)].has_sim_collider) {
                    w.island_order.push_back(cpi);
                    total_manifolds += cp.nman;
                    w.islands[isl_index].manifold_count += cp.nman;
                    if (in_island[size_t(other)]) continue;
                    stack.push_back(other);
                    in_island[size_t(other)] = 1;
                }
            }
            // the body's joints (PhysicsWorld.cpp:822-844)
            for (int j : w.bodies[size_t(b)].joints) {
                JointH& J = w.joints[size_t(j)];
                if (J.in_island) continue;
                J.in_island = true;
                const int other = J.b1 == b ? J.b2 : J.b1;
                if (in_island[size_t(other)]) continue;
                stack.push_back(other);
                in_island[size_t(other)] = true;
            }
        }
        for (int sb : statics) in_island[size_t(sb)] = 0;
        statics.clear();
    }
    w.nm = total_manifolds;
    w.np = 0;
    for (uint32_t m = 0; m < w.island_order.size(); m++) w.np += w.cpairs[w.island_order[m]].k;
    // PhysicsWorld::enableDisableJoints (:363-393): a joint is enabled while
    // one of its bodies is
    if (!w.joints.empty()) {
        const std::vector<int> order = w.jcomp.at;
        for (int j : order) {
            const JointH& J = w.joints[size_t(j)];
            const bool dis = !w.bcomp.enabled(J.b1) && !w.bcomp.enabled(J.b2);
            if (w.jcomp.enabled(j) == !dis) continue;
            w.jcomp.set_disabled(j, dis);
            joint_type_comps(w, J.type).set_disabled(j, dis);
        }
    }
    // the enabled joints island by island: ball-and-socket, fixed, hinge then
    // slider, each in component order (the order the constraint solver visits
    // them, ConstraintSolverSystem.cpp:60-113)
    w.jlist.clear();
    w.isl_jstart.assign(w.islands.size(), 0);
    w.isl_jcount.assign(w.islands.size(), 0);
    if (!w.joints.empty()) {
        // (joint, island) in visiting order, then a stable counting sort by island
        std::vector<int2>& jv = w.jvisit;
        jv.clear();
        for (rp3dg::order::Comps* cmp : {&w.bscomp, &w.fcomp, &w.hcomp, &w.scomp})
            for (uint32_t s = 0; s < cmp->n_enabled; s++) {
                const int j = cmp->at[s];
                const JointH& J = w.joints[size_t(j)];
                const int isl = w.bodies[size_t(J.b1)].type != RP3DG_BODY_STATIC ? w.b_island[size_t(J.b1)]
                                                                                  : w.b_island[size_t(J.b2)];
                if (isl >= 0) {
                    jv.push_back(make_int2(j, isl));
                    w.isl_jcount[size_t(isl)]++;
                }
            }
        uint32_t run = 0;
        for (size_t i = 0; i < w.islands.size(); i++) {
            w.isl_jstart[i] = run;
            run += w.isl_jcount[i];
        }
        w.jlist.resize(jv.size());
        std::vector<uint32_t>& fill = w.jfill;
        fill.assign(w.isl_jstart.begin(), w.isl_jstart.end());
        for (const int2 e : jv) {
            const JointH& J = w.joints[size_t(e.x)];
            const int flags = (w.bodies[size_t(J.b1)].type == RP3DG_BODY_DYNAMIC ? 1 : 0) |
                              (w.bodies[size_t(J.b2)].type == RP3DG_BODY_DYNAMIC ? 2 : 0);
            // rows filled in fill_manifolds (after the row sync)
            w.jlist[fill[size_t(e.y)]++] = make_int4(int(w.jbase) + e.x, J.b1, J.b2, flags);
        }
    }
}

// createContacts' packing (CollisionDetectionSystem.cpp:906-975) and the
// warm-start sources of initContactsWithPreviousOnes (:1069-1160).
void fill_manifolds(Group* g, WorldH& w) {
    uint32_t pt = w.pt_base;
    uint32_t gm = w.man_base;
    for (uint32_t o = 0; o < w.island_order.size(); o++) {
        ContactPairH& cp = w.cpairs[w.island_order[o]];
        cp.manifold = gm;
        cp.point = pt;
        const int4 ids = make_int4(int(w.b0) + w.bcomp.slot[size_t(cp.b1)], int(w.b0) + w.bcomp.slot[size_t(cp.b2)],
                                   int(w.c0) + w.ccomp.slot[size_t(cp.c1)], int(w.c0) + w.ccomp.slot[size_t(cp.c2)]);
        int4 prev = make_int4(-1, 0, 0, 0);
        uint32_t pi = 0;
        if (w.prev_map.get(cp.id, pi) && w.prev_cpairs[pi].in_island) {
            const ContactPairH& pc = w.prev_cpairs[pi];
            prev = make_int4(int(pc.manifold), int(pc.nman), int(pc.point), int(pc.k));
        }
        if (!cp.concave) {
            uint32_t a = 0;
            while (cp.item >= g->batch_start[a + 1]) a++;
            const uint32_t s0 = g->batch_start[a];
            g->h_mids[gm] = ids;
            g->h_msrc[gm] = make_int4(int(cp.item - s0), int(g->batch_start[a + 1] - s0), int(s0), int(pt));
            g->h_mprev[gm] = prev;
            gm++;
            pt += cp.k;
        } else {
            for (uint32_t m = 0; m < cp.nman; m++) {
                const uint32_t km = (cp.npts >> (8 * m)) & 0xffu;
                g->h_mids[gm] = ids;
                g->h_msrc[gm] = make_int4(int(cp.item * HF_OUT_POINTS + 4 * m), -1, int(km), int(pt));
                g->h_mprev[gm] = prev;
                gm++;
                pt += km;
            }
        }
    }
    for (uint32_t i = 0; i < w.islands.size(); i++) {
        g->h_istart[w.isl_base + i] = w.man_base + w.islands[i].manifold_start;
        g->h_icount[w.isl_base + i] = w.islands[i].manifold_count;
        g->h_ijstart[w.isl_base + i] = w.jl_base + w.isl_jstart[i];
        g->h_ijcount[w.isl_base + i] = w.isl_jcount[i];
    }
    for (size_t k = 0; k < w.jlist.size(); k++) {
        int4 e = w.jlist[k];
        e.y = int(w.b0) + w.bcomp.slot[size_t(e.y)];
        e.z = int(w.b0) + w.bcomp.slot[size_t(e.z)];
        g->h_jlist[w.jl_base + k] = e;
    }
    // islands with joints and their bodies' rows (the joints' position correction)
    w.ji_isl.clear();
    w.ji_bcount.clear();
    w.ji_rows.clear();
    if (!w.jlist.empty())
        for (uint32_t i = 0; i < w.islands.size(); i++) {
            if (!w.isl_jcount[i]) continue;
            w.ji_isl.push_back(w.isl_base + i);
            const uint32_t r0 = uint32_t(w.ji_rows.size());
            for (uint32_t ib = w.islands[i].body_start; ib < w.islands[i].body_start + w.islands[i].body_count; ib++) {
                const int b = w.isl_bodies[ib];
                if (w.bodies[size_t(b)].type != RP3DG_BODY_STATIC)
                    w.ji_rows.push_back(int32_t(w.b0) + w.bcomp.slot[size_t(b)]);
            }
            w.ji_bcount.push_back(uint32_t(w.ji_rows.size()) - r0);
        }
    // computeMapPreviousContactPairs for the next step
    w.prev_map.clear_for(w.cpairs.size());
    for (uint32_t i = 0; i < w.cpairs.size(); i++) w.prev_map.put(w.cpairs[i].id, i);
}

// BroadPhaseSystem::updateColliders' reinsertions (enabled colliders in
// component order) and PhysicsWorld::updateSleepingBodies (:871-926).
void colliders_and_sleep(Group* g, WorldH& w, float dt, const uint8_t* h_moved, const float4* h_fmin,
                         const float4* h_fmax, const uint8_t* h_fast) {
    uint32_t nmoved = 0;
    for (uint32_t s = 0; s < w.ccomp.n_enabled; s++) {
        const uint32_t r = w.c0 + s;
        if (!h_moved[r]) continue;
        const int c = w.ccomp.at[s];
        Box box;
        box.mn[0] = h_fmin[r].x; box.mn[1] = h_fmin[r].y; box.mn[2] = h_fmin[r].z;
        box.mx[0] = h_fmax[r].x; box.mx[1] = h_fmax[r].y; box.mx[2] = h_fmax[r].z;
        const int bp = w.colliders[size_t(c)].bp;
        if (g->dev_tree) {
            // the device tree reinserts (reinsert_on_device); the host keeps the leaf's box
            w.tree.nodes[size_t(bp)].box = box;
            w.tree_stale = true;
        } else {
            w.tree.reinsert(bp, box);
        }
        add_moved(w, c);
        nmoved++;
    }
    w.stats.moved_colliders = nmoved;
    w.slept.clear();
    if (g->set.sleeping_enabled) {
        // the velocity condition by body id (world_sleep_fast, rows in the
        // device order before any body falls asleep)
        std::vector<uint8_t>& fast = w.sleep_fast;
        fast.resize(w.nb);
        for (uint32_t s = 0; s < w.nb; s++) fast[size_t(w.dev_body_at[s])] = h_fast[w.b0 + s];
        for (const IslandH& isl : w.islands) {
            float min_sleep = 3.40282347e+38f;
            for (uint32_t ib = isl.body_start; ib < isl.body_start + isl.body_count; ib++) {
                const int b = w.isl_bodies[ib];
                BodyH& B = w.bodies[size_t(b)];
                if (B.type == RP3DG_BODY_STATIC) continue;
                if (fast[size_t(b)] || !B.allowed_sleep) {
                    B.sleep_time = 0.0f;
                    min_sleep = 0.0f;
                } else {
                    B.sleep_time += dt;
                    if (B.sleep_time < min_sleep) min_sleep = B.sleep_time;
                }
            }
            if (min_sleep >= g->set.time_before_sleep)
                for (uint32_t ib = isl.body_start; ib < isl.body_start + isl.body_count; ib++)
                    set_sleeping(g, w, w.isl_bodies[ib], true);
        }
    }
    // (collidingInPreviousFrame moves at the next step's item loops)
    w.prev_cpairs.swap(w.cpairs);
    w.stats.disabled_pairs = uint32_t(w.disabled.size() + w.concave_dis.size());
    w.stats.enabled_bodies = w.bcomp.n_enabled;
}

int ensure_items(Group* g, size_t n) {
    if (n <= g->cap_items) return 0;
    size_t c = std::max<size_t>(n, g->cap_items * 2);
    c = std::max<size_t>(c, 256);
    cudaFree(g->d_items); cudaFree(g->d_s1); cudaFree(g->d_s2); cudaFree(g->d_p1); cudaFree(g->d_r1);
    cudaFree(g->d_p2); cudaFree(g->d_r2); cudaFree(g->d_rep); cudaFree(g->d_coll); cudaFree(g->d_nct);
    cudaFree(g->d_cache); cudaFree(g->d_nd); cudaFree(g->d_l1); cudaFree(g->d_l2);
    cudaError_t e = cudaSuccess;
    auto M = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, b); };
    M((void**)&g->d_items, c * 16); M((void**)&g->d_s1, c * 4); M((void**)&g->d_s2, c * 4);
    M((void**)&g->d_p1, c * 16); M((void**)&g->d_r1, c * 16); M((void**)&g->d_p2, c * 16); M((void**)&g->d_r2, c * 16);
    M((void**)&g->d_rep, c); M((void**)&g->d_coll, c); M((void**)&g->d_nct, c);
    M((void**)&g->d_cache, c * 16);
    M((void**)&g->d_nd, c * 16 * MAXC); M((void**)&g->d_l1, c * 16 * MAXC); M((void**)&g->d_l2, c * 16 * MAXC);
    if (e != cudaSuccess) { g->cap_items = 0; return wcuda(g, e, "cudaMalloc(narrow-phase step buffers)"); }
    g->cap_items = c;
    if (host_grow(&g->h_items, &g->cap_hitems, c) || host_grow(&g->h_out, &g->cap_hout, 2 * c))
        return wfail(g, RP3DG_ENOMEM, "cudaMallocHost(step staging)");
    return 0;
}

int ensure_pool(Group* g, size_t reserve = 0) {
    const size_t need = std::max<size_t>(g->cache_next.load(), reserve);
    if (need <= g->cap_pool) return 0;
    size_t c = std::max<size_t>(need, g->cap_pool * 2);
    c = std::max<size_t>(c, 1024);
    rp3dg_lastframe* np = nullptr;
    cudaError_t e = cudaMalloc(&np, c * sizeof(rp3dg_lastframe));
    if (e != cudaSuccess) return wcuda(g, e, "cudaMalloc(cache pool)");
    if (g->pool && g->cap_pool)
        cudaMemcpyAsync(np, g->pool, g->cap_pool * sizeof(rp3dg_lastframe), cudaMemcpyDeviceToDevice, g->stream);
    cudaStreamSynchronize(g->stream);
    cudaFree(g->pool);
    g->pool = np;
    g->cap_pool = c;
    return 0;
}

int ensure_small(Group* g, size_t n) { return dev_grow(&g->d_small, &g->cap_small, n) ? wfail(g, RP3DG_ENOMEM, "cudaMalloc(small)") : 0; }

// Per-item arrays of the convex vs concave pairs (pinned staging + device).
int ensure_hitems(Group* g, size_t n) {
    if (n <= g->cap_hitem && g->h_hitems) return 0;
    const size_t c = std::max<size_t>(std::max<size_t>(n, g->cap_hitem * 2), 64);
    cudaFreeHost(g->h_hitems); cudaFreeHost(g->h_hrect); cudaFreeHost(g->h_hstart); cudaFreeHost(g->h_hpstart);
    cudaFreeHost(g->h_hprect); cudaFreeHost(g->h_hbatch); cudaFreeHost(g->h_hout);
    cudaFree(g->d_hitems); cudaFree(g->d_hrect); cudaFree(g->d_hstart); cudaFree(g->d_hpstart); cudaFree(g->d_hprect);
    cudaFree(g->d_hbatch); cudaFree(g->d_hout); cudaFree(g->d_hond); cudaFree(g->d_hol1); cudaFree(g->d_hol2);
    g->h_hitems = g->h_hrect = g->h_hprect = g->h_hbatch = nullptr;
    g->h_hstart = nullptr; g->h_hpstart = nullptr; g->h_hout = nullptr;
    g->d_hitems = g->d_hrect = g->d_hprect = g->d_hbatch = nullptr;
    g->d_hstart = nullptr; g->d_hpstart = nullptr; g->d_hout = nullptr;
    g->d_hond = g->d_hol1 = g->d_hol2 = nullptr;
    g->cap_hitem = 0;
    bool ok = true;
    auto H = [&](void** p, size_t b) { if (ok && cudaMallocHost(p, b) != cudaSuccess) ok = false; };
    auto D = [&](void** p, size_t b) { if (ok && cudaMalloc(p, b) != cudaSuccess) ok = false; };
    H((void**)&g->h_hitems, c * 16); H((void**)&g->h_hrect, c * 16); H((void**)&g->h_hstart, (c + 1) * 4);
    H((void**)&g->h_hpstart, c * 4); H((void**)&g->h_hprect, c * 16); H((void**)&g->h_hbatch, c * 16);
    H((void**)&g->h_hout, c * 6);
    D((void**)&g->d_hitems, c * 16); D((void**)&g->d_hrect, c * 16); D((void**)&g->d_hstart, (c + 1) * 4);
    D((void**)&g->d_hpstart, c * 4); D((void**)&g->d_hprect, c * 16); D((void**)&g->d_hbatch, c * 16);
    D((void**)&g->d_hout, c * 6);
    D((void**)&g->d_hond, c * HF_OUT_POINTS * 16); D((void**)&g->d_hol1, c * HF_OUT_POINTS * 16);
    D((void**)&g->d_hol2, c * HF_OUT_POINTS * 16);
    if (!ok) return wfail(g, RP3DG_ENOMEM, "allocation of concave-pair arrays");
    g->cap_hitem = c;
    return 0;
}

// Per-test arrays of the triangle tests; the record buffer of this step
// (the previous step's buffer is kept as it is).
int ensure_htests(Group* g, size_t n) {
    n = std::max<size_t>(n, 1);
    if (dev_grow(&g->d_tcache[g->cur_tc], &g->cap_hc[g->cur_tc], n) ||
        dev_grow(&g->d_ttri[g->cur_tc], &g->cap_ttri[g->cur_tc], n))
        return wfail(g, RP3DG_ENOMEM, "cudaMalloc(triangle records)");
    if (n <= g->cap_htest) return 0;
    const size_t c = std::max<size_t>(std::max<size_t>(n, g->cap_htest * 2), 256);
    cudaFree(g->d_ts1); cudaFree(g->d_ts2); cudaFree(g->d_tp1); cudaFree(g->d_tr1); cudaFree(g->d_tp2);
    cudaFree(g->d_tr2); cudaFree(g->d_trep); cudaFree(g->d_tcoll); cudaFree(g->d_tnct); cudaFree(g->d_tmid);
    cudaFree(g->d_tnd); cudaFree(g->d_tl1); cudaFree(g->d_tl2); cudaFree(g->d_tri);
    g->cap_htest = 0;
    cudaError_t e = cudaSuccess;
    auto M = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, b); };
    M((void**)&g->d_ts1, c * 4); M((void**)&g->d_ts2, c * 4);
    M((void**)&g->d_tp1, c * 16); M((void**)&g->d_tr1, c * 16); M((void**)&g->d_tp2, c * 16); M((void**)&g->d_tr2, c * 16);
    M((void**)&g->d_trep, c); M((void**)&g->d_tcoll, c); M((void**)&g->d_tnct, c); M((void**)&g->d_tmid, c * MAXC);
    M((void**)&g->d_tnd, c * 16 * MAXC); M((void**)&g->d_tl1, c * 16 * MAXC); M((void**)&g->d_tl2, c * 16 * MAXC);
    M((void**)&g->d_tri, c * 16 * rp3dg::TRI_REC);
    if (e != cudaSuccess) return wcuda(g, e, "cudaMalloc(triangle tests)");
    g->cap_htest = c;
    return 0;
}

// Run f(world index) for every world on the group's host threads.
template <class F>
void for_worlds(Group* g, F f) {
    const int n = int(g->worlds.size());
    if (g->nthreads <= 1 || n <= 1) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
#pragma omp parallel for schedule(dynamic, 4) num_threads(g->nthreads)
    for (int i = 0; i < n; i++) f(i);
}

// ---- device trees of a world group

// Nodes of a world's tree that its device copy holds: a reinsertion frees
// one node (its leaf's parent) and then takes that same node back, so a tree
// never grows after its colliders were added and only the nodes below the
// first never-used one (nodes in use, plus the free list's head) are ever
// read or written; the rest of the host array stays as it is.
int device_tree_nodes(const rp3dg::order::Tree& t) {
    return std::min<int>(int(t.nodes.size()), t.nb_nodes + 1);
}

// Copies every world's host tree into the group's device pool.
int upload_trees(Group* g) {
    const size_t nw = g->worlds.size();
    g->tree_base.assign(nw, 0);
    size_t total = 0;
    for (size_t k = 0; k < nw; k++) {
        g->tree_base[k] = uint32_t(total);
        total += size_t(device_tree_nodes(g->worlds[k].tree));
    }
    if (total >= (size_t(1) << 31)) return wfail(g, RP3DG_EINVAL, "world group trees too large for the device pool");
    cudaFree(g->d_tree);
    cudaFree(g->d_tree_base);
    cudaFree(g->d_tree_hdr);
    cudaFree(g->d_tree_rows);
    g->d_tree = nullptr;
    g->d_tree_base = nullptr;
    g->d_tree_hdr = nullptr;
    g->d_tree_rows = nullptr;
    if (cudaMalloc(&g->d_tree, std::max<size_t>(total, 1) * sizeof(TreeNode)) != cudaSuccess ||
        cudaMalloc(&g->d_tree_base, std::max<size_t>(nw, 1) * 4) != cudaSuccess ||
        cudaMalloc(&g->d_tree_hdr, std::max<size_t>(nw, 1) * sizeof(int4)) != cudaSuccess ||
        cudaMalloc(&g->d_tree_rows, std::max<size_t>(nw, 1) * sizeof(uint2)) != cudaSuccess ||
        !pair_grow(&g->h_tcnt, &g->d_tcnt, &g->cap_tcnt, 4))
        return wfail(g, RP3DG_ENOMEM, "cudaMalloc(device trees)");
    if (!g->ev_step_copy && cudaEventCreateWithFlags(&g->ev_step_copy, cudaEventDisableTiming) != cudaSuccess)
        return wfail(g, RP3DG_ECUDA, "cudaEventCreate(step copies)");
    std::vector<TreeNode> nodes(total);
    std::vector<int4> hdr(nw);
    std::vector<uint2> rows(nw);
    for (size_t k = 0; k < nw; k++) {
        const rp3dg::order::Tree& t = g->worlds[k].tree;
        const int n = device_tree_nodes(t);
        std::copy(t.nodes.begin(), t.nodes.begin() + n, nodes.begin() + g->tree_base[k]);
        hdr[k] = make_int4(t.root, t.free_id, t.nb_nodes, n);
        rows[k] = make_uint2(g->worlds[k].c0, g->worlds[k].nc);
        g->worlds[k].tree_stale = false;
    }
    cudaStream_t st = g->stream;
    cudaMemcpyAsync(g->d_tree, nodes.data(), total * sizeof(TreeNode), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(g->d_tree_base, g->tree_base.data(), nw * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(g->d_tree_hdr, hdr.data(), nw * sizeof(int4), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(g->d_tree_rows, rows.data(), nw * sizeof(uint2), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(g->d_tcnt, 0, 16, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? 0 : wcuda(g, e, "upload of the device trees");
}

// Brings world k's host tree up to date with its device tree (before a host
// reader of the inner nodes: world raycasts, switching the device trees off).
int download_tree(Group* g, uint32_t k) {
    WorldH& w = g->worlds[k];
    if (!g->dev_tree || !w.tree_stale) return 0;
    cudaStream_t st = g->stream;
    int4 h;
    cudaMemcpyAsync(&h, g->d_tree_hdr + k, sizeof(int4), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return wcuda(g, e, "download of a device tree");
    if (h.w != device_tree_nodes(w.tree) || h.z != w.tree.nb_nodes)
        return wfail(g, RP3DG_EINVAL, "device tree size changed");
    cudaMemcpyAsync(w.tree.nodes.data(), g->d_tree + g->tree_base[k], size_t(h.w) * sizeof(TreeNode),
                    cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return wcuda(g, e, "download of a device tree");
    w.tree.root = h.x;
    w.tree.free_id = h.y;
    w.tree.nb_nodes = h.z;
    w.tree_stale = false;
    return 0;
}

// Queues the reinsertions of every world's moved colliders on the device
// trees (the step's moved flags and fat AABBs by row, rows as the last row
// sync left them).
int reinsert_on_device(Group* g, const uint8_t* moved, const float4* fmin, const float4* fmax) {
    const size_t nw = g->worlds.size();
    if (!nw) return 0;
    TreeReinsertArgs a{};
    a.nworlds = uint32_t(nw);
    a.pool = g->d_tree;
    a.base = g->d_tree_base;
    a.hdr = g->d_tree_hdr;
    a.rows = g->d_tree_rows;
    a.enabled = g->c_en;
    a.moved = moved;
    a.leaf = g->c_leaf;
    a.fmin = fmin;
    a.fmax = fmax;
    a.error = g->d_tcnt + 2;
    world_tree_reinsert<<<uint32_t((nw * 32 + 127) / 128), 128, 0, g->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : wcuda(g, e, "tree reinsertion launch");
}

// The moved colliders' queries of every world on the device trees: world
// k's leaves of its i-th moved collider are h_tleaves[h_tpos[q_off + i]].
int tree_queries_group(Group* g) {
    const size_t nw = g->worlds.size();
    for_worlds(g, [&](int k) {
        WorldH& w = g->worlds[size_t(k)];
        w.moved.to_array(w.q_shapes);
        w.moved.clear();
    });
    size_t nq = 0;
    for (WorldH& w : g->worlds) {
        w.q_off = uint32_t(nq);
        nq += w.q_shapes.size();
    }
    if (!pair_grow(&g->h_gq, &g->d_gq, &g->cap_gq, std::max<size_t>(nq, 1)) ||
        !pair_grow(&g->h_tpos, &g->d_tpos, &g->cap_tpos, std::max<size_t>(nq, 1)) ||
        !pair_grow(&g->h_tcnt, &g->d_tcnt, &g->cap_tcnt, 4) ||
        !pair_grow(&g->h_tleaves, &g->d_tleaves, &g->cap_tleaves, 8 * nq))
        return wfail(g, RP3DG_ENOMEM, "cudaMalloc(tree queries)");
    for_worlds(g, [&](int k) {
        const WorldH& w = g->worlds[size_t(k)];
        for (size_t i = 0; i < w.q_shapes.size(); i++) g->h_gq[w.q_off + i] = make_int2(k, w.q_shapes[i]);
    });
    cudaStream_t st = g->stream;
    if (nq) cudaMemcpyAsync(g->d_gq, g->h_gq, nq * sizeof(int2), cudaMemcpyHostToDevice, st);
    for (int attempt = 0; attempt < 2; attempt++) {
        cudaMemsetAsync(g->d_tcnt, 0, 8, st);
        if (nq)
            world_tree_query_group<<<blocks(uint32_t(nq)), 128, 0, st>>>(
                g->d_tree, g->d_tree_base, g->d_tree_hdr, g->d_gq, uint32_t(nq), g->d_tpos, g->d_tleaves,
                uint32_t(g->cap_tleaves), g->d_tcnt, g->d_tcnt + 1);
        cudaMemcpyAsync(g->h_tcnt, g->d_tcnt, 16, cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return wcuda(g, e, "tree queries");
        const uint32_t total = g->h_tcnt[0], flags = g->h_tcnt[1];
        if (g->h_tcnt[2]) return wfail(g, RP3DG_ECUDA, "device tree reinsertion failed");
        if (flags & 1u) return wfail(g, RP3DG_ECUDA, "device tree query: stack overflow or leaf out of range");
        if (flags & 2u) {
            if (attempt || !pair_grow(&g->h_tleaves, &g->d_tleaves, &g->cap_tleaves, size_t(total) + 1024))
                return wfail(g, RP3DG_ENOMEM, "cudaMalloc(tree query leaves)");
            continue;
        }
        if (nq) cudaMemcpyAsync(g->h_tpos, g->d_tpos, nq * sizeof(int2), cudaMemcpyDeviceToHost, st);
        if (total) cudaMemcpyAsync(g->h_tleaves, g->d_tleaves, size_t(total) * 4, cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? 0 : wcuda(g, e, "tree queries");
    }
    return wfail(g, RP3DG_ECUDA, "tree queries");
}

// Host copies of the per-row tables (pinned), kept current world by world.
void world_tables(Group* g, WorldH& w) {
    for (uint32_t r = 0; r < w.nb; r++) {
        g->t_grav[w.b0 + r] = w.gravity[size_t(w.bcomp.at[r])];
        g->t_ben[w.b0 + r] = r < w.bcomp.n_enabled ? 1 : 0;
    }
    for (uint32_t r = 0; r < w.nc; r++) {
        const ColliderH& C = w.colliders[size_t(w.ccomp.at[r])];
        g->t_cbody[w.c0 + r] = int32_t(w.b0) + w.bcomp.slot[size_t(C.body)];
        g->t_cshape[w.c0 + r] = C.shape;
        g->t_cleaf[w.c0 + r] = C.bp;
        g->t_cat[w.c0 + r] = C.category;
        g->t_mask[w.c0 + r] = C.mask;
        g->t_cen[w.c0 + r] = r < w.ccomp.n_enabled ? 1 : 0;
    }
}

int ensure_tables(Group* g) {
    if (g->t_grav) return 0;
    const size_t nb = std::max<uint32_t>(g->NB, 1), nc = std::max<uint32_t>(g->NC, 1);
    if (cudaMallocHost(&g->t_grav, nb) || cudaMallocHost(&g->t_ben, nb) || cudaMallocHost(&g->t_cen, nc) ||
        cudaMallocHost(&g->t_cbody, nc * 4) || cudaMallocHost(&g->t_cshape, nc * 4) || cudaMallocHost(&g->t_cleaf, nc * 4) ||
        cudaMallocHost(&g->t_cat, nc * 2) || cudaMallocHost(&g->t_mask, nc * 2) ||
        cudaMallocHost(&g->t_bperm, nb * 4) || cudaMallocHost(&g->t_cperm, nc * 4))
        return wfail(g, RP3DG_ENOMEM, "cudaMallocHost(row tables)");
    for (uint32_t r = 0; r < g->NB; r++) g->t_bperm[r] = int32_t(r);
    for (uint32_t r = 0; r < g->NC; r++) g->t_cperm[r] = int32_t(r);
    return 0;
}

// Device rows follow the host's component order.  Worlds whose order changed
// (a sleep, wake or type change moved components) or whose enabled counts
// changed get their permutation segment and table rows rebuilt (in
// parallel); one permutation kernel and one upload per table then cover all
// rows.
int sync_rows(Group* g) {
    int rc = ensure_tables(g);
    if (rc) return rc;
    std::atomic<int> bchg{0}, cchg{0}, tchg{0};
    for_worlds(g, [&](int k) {
        WorldH& w = g->worlds[size_t(k)];
        const bool bo = w.dev_body_at != w.bcomp.at, co = w.dev_col_at != w.ccomp.at;
        const bool en = w.dev_nb_en != w.bcomp.n_enabled || w.dev_nc_en != w.ccomp.n_enabled;
        if (bo) {
            std::vector<int32_t> inv(w.nb);
            for (uint32_t r = 0; r < w.nb; r++) inv[size_t(w.dev_body_at[r])] = int32_t(r);
            for (uint32_t r = 0; r < w.nb; r++) g->t_bperm[w.b0 + r] = int32_t(w.b0) + inv[size_t(w.bcomp.at[r])];
            w.dev_body_at = w.bcomp.at;
            bchg = 1;
        }
        if (co) {
            std::vector<int32_t> inv(w.nc);
            for (uint32_t r = 0; r < w.nc; r++) inv[size_t(w.dev_col_at[r])] = int32_t(r);
            for (uint32_t r = 0; r < w.nc; r++) g->t_cperm[w.c0 + r] = int32_t(w.c0) + inv[size_t(w.ccomp.at[r])];
            w.dev_col_at = w.ccomp.at;
            cchg = 1;
        }
        if (bo || co || en || g->tables_dirty) {
            world_tables(g, w);
            w.dev_nb_en = w.bcomp.n_enabled;
            w.dev_nc_en = w.ccomp.n_enabled;
            tchg = 1;
        }
    });
    cudaStream_t st = g->stream;
    if (bchg) {
        if (ensure_small(g, g->NB)) return RP3DG_ENOMEM;
        cudaMemcpyAsync(g->d_small, g->t_bperm, size_t(g->NB) * 4, cudaMemcpyHostToDevice, st);
        PermArgs a{};
        a.n = g->NB;
        a.perm = g->d_small;
        const int s = g->cur_b, d = 1 - s;
        for (int c = 0; c < BC_NCOL; c++) a.col[a.ncol++] = PermCol{g->bcol[s][c], g->bcol[d][c], 1};
        a.col[a.ncol++] = PermCol{g->biiw[s], g->biiw[d], 3};
        world_permute<<<blocks(g->NB), 128, 0, st>>>(a);
        g->cur_b = d;
    }
    if (cchg) {
        // the small buffer holds the body permutation until its kernel ran
        cudaStreamSynchronize(st);
        if (ensure_small(g, g->NC)) return RP3DG_ENOMEM;
        cudaMemcpyAsync(g->d_small, g->t_cperm, size_t(g->NC) * 4, cudaMemcpyHostToDevice, st);
        PermArgs a{};
        a.n = g->NC;
        a.perm = g->d_small;
        const int s = g->cur_c, d = 1 - s;
        for (int c = 0; c < CC_NCOL; c++) a.col[a.ncol++] = PermCol{g->ccol[s][c], g->ccol[d][c], 1};
        world_permute<<<blocks(g->NC), 128, 0, st>>>(a);
        g->cur_c = d;
    }
    if (tchg) {
        cudaMemcpyAsync(g->bgrav, g->t_grav, g->NB, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->b_en, g->t_ben, g->NB, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->c_en, g->t_cen, g->NC, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->c_body, g->t_cbody, size_t(g->NC) * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->c_leaf, g->t_cleaf, size_t(g->NC) * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->c_shape, g->t_cshape, size_t(g->NC) * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->c_cat, g->t_cat, size_t(g->NC) * 2, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->c_mask, g->t_mask, size_t(g->NC) * 2, cudaMemcpyHostToDevice, st);
    }
    g->tables_dirty = false;
    // the host buffers are rewritten by the next sync: wait for the copies
    if (bchg || cchg || tchg) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return wcuda(g, e, "row sync");
        if (bchg)
            for_worlds(g, [&](int k) {
                const WorldH& w = g->worlds[size_t(k)];
                for (uint32_t r = 0; r < w.nb; r++) g->t_bperm[w.b0 + r] = int32_t(w.b0 + r);
            });
        if (cchg)
            for_worlds(g, [&](int k) {
                const WorldH& w = g->worlds[size_t(k)];
                for (uint32_t r = 0; r < w.nc; r++) g->t_cperm[w.c0 + r] = int32_t(w.c0 + r);
            });
    }
    return 0;
}

// DebugRenderer at the end of PhysicsWorld::update (PhysicsWorld.cpp:248-303):
// the contact primitives of DebugRenderer::onContact, from the contact pairs
// of the update that are not triggers (CollisionCallback.cpp:84-103), then
// computeDebugRenderingPrimitives over the bodies in creation order
// (DebugRenderer.cpp:482-527), every world after the other.  The host lays
// out the offsets; debug.cu writes the primitives.
int debug_primitives(Group* g) {
    const uint32_t items = g->debug_items;
    if (!items) return 0;
    const bool cpt = (items & RP3DG_DEBUG_CONTACT_POINT) != 0, cno = (items & RP3DG_DEBUG_CONTACT_NORMAL) != 0;
    std::vector<rp3dg::DebugJob> jobs;
    std::vector<int4> points;
    std::unordered_map<int32_t, std::vector<uint32_t>> faces;
    std::vector<rp3dg::CmDesc> cms;
    rp3dg::get_cmeshes(g->ctx, &cms);
    uint32_t nl = 0, nt = 0;
    for (WorldH& w : g->worlds) {
        w.dbg_line0 = nl;
        w.dbg_tri0 = nt;
        std::vector<int32_t> row_of(w.nc);
        for (uint32_t r = 0; r < w.nc; r++) row_of[size_t(w.dev_col_at[r])] = int32_t(w.c0 + r);
        if (cpt || cno)
            for (const ContactPairH& c : w.prev_cpairs) {
                if (c.trigger || !c.in_island) continue;
                for (uint32_t i = 0; i < c.k; i++) {
                    points.push_back(make_int4(row_of[size_t(c.c1)], int(c.point + i), int(nl), int(nt)));
                    nl += cno ? 1u : 0u;
                    nt += cpt ? rp3dg::DEBUG_SPHERE_TRIS : 0u;
                }
            }
        for (uint32_t b = 0; b < w.nb; b++) {
            if (!w.body_debug[b]) continue;
            for (int c : w.bodies[b].colliders) {
                const int si = w.colliders[size_t(c)].shape;
                const rp3dg_shape& sh = g->shapes[size_t(si)];
                const uint32_t* fc = nullptr;
                uint32_t nf = 0, hc = 0, hr = 0, cv = 0, ct = 0;
                if (sh.kind == RP3DG_SHAPE_CONVEX_MESH) {
                    auto it = faces.find(sh.mesh);
                    if (it == faces.end()) {
                        std::vector<uint32_t> v;
                        if (rp3dg::get_mesh_face_counts(g->ctx, sh.mesh, &v))
                            return wfail(g, RP3DG_EINVAL, "debug rendering: unknown convex mesh");
                        it = faces.emplace(sh.mesh, std::move(v)).first;
                    }
                    fc = it->second.data();
                    nf = uint32_t(it->second.size());
                } else if (sh.kind == RP3DG_SHAPE_HEIGHTFIELD) {
                    rp3dg::HfDesc h;
                    if (rp3dg::get_heightfield(g->ctx, sh.mesh, &h))
                        return wfail(g, RP3DG_EINVAL, "debug rendering: unknown height field");
                    hc = h.ncol;
                    hr = h.nrow;
                } else if (sh.kind == RP3DG_SHAPE_CONCAVE_MESH) {
                    if (sh.mesh < 0 || uint32_t(sh.mesh) >= g->n_cm)
                        return wfail(g, RP3DG_EINVAL, "debug rendering: unknown concave mesh");
                    cv = cms[size_t(sh.mesh)].nv;
                    ct = cms[size_t(sh.mesh)].nt;
                }
                uint32_t l = 0, t = 0;
                rp3dg::debug_collider_counts(items, sh.kind, fc, nf, hc, hr, cv, ct, &l, &t);
                if (l || t) jobs.push_back(rp3dg::DebugJob{row_of[size_t(c)], si, nl, nt});
                nl += l;
                nt += t;
            }
        }
        w.dbg_nl = nl - w.dbg_line0;
        w.dbg_nt = nt - w.dbg_tri0;
    }
    if (dev_grow(&g->d_dbg_lines, &g->cap_dbg_lines, std::max<size_t>(nl, 1)) ||
        dev_grow(&g->d_dbg_tris, &g->cap_dbg_tris, std::max<size_t>(nt, 1)) ||
        dev_grow(&g->d_dbg_jobs, &g->cap_dbg_jobs, std::max<size_t>(jobs.size(), 1)) ||
        dev_grow(&g->d_dbg_points, &g->cap_dbg_points, std::max<size_t>(points.size(), 1)))
        return wfail(g, RP3DG_ENOMEM, "cudaMalloc(debug primitives)");
    if (jobs.empty() && points.empty()) return 0;
    cudaStream_t st = g->stream;
    if (!jobs.empty())
        cudaMemcpyAsync(g->d_dbg_jobs, jobs.data(), jobs.size() * sizeof(rp3dg::DebugJob), cudaMemcpyHostToDevice, st);
    if (!points.empty())
        cudaMemcpyAsync(g->d_dbg_points, points.data(), points.size() * sizeof(int4), cudaMemcpyHostToDevice, st);
    rp3dg::DebugArgs a{};
    a.items = items;
    a.n_jobs = uint32_t(jobs.size());
    a.jobs = g->d_dbg_jobs;
    a.wpos = g->ccol[g->cur_c][CC_WPOS];
    a.wori = g->ccol[g->cur_c][CC_WORI];
    a.fmin = g->ccol[g->cur_c][CC_FMIN];
    a.fmax = g->ccol[g->cur_c][CC_FMAX];
    rp3dg::get_shape_device(g->ctx, &a.shapes, &a.bounds);
    rp3dg::get_mesh_arena_device(g->ctx, &a.mesh_words);
    a.hf = g->d_hf;
    a.cm = g->d_cm;
    a.n_points = uint32_t(points.size());
    a.points = g->d_dbg_points;
    a.snap_wpos = g->d_dbg_snap;
    a.snap_wori = g->d_dbg_snap ? g->d_dbg_snap + g->NC : nullptr;
    const ContactBuf& B = g->cbuf[1 - g->cur_cb];
    a.nd = B.nd;
    a.l1 = B.l1;
    a.lines = g->d_dbg_lines;
    a.tris = g->d_dbg_tris;
    rp3dg::make_debug_trig(&a.trig);
    cudaError_t e = rp3dg::launch_debug(a, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? 0 : wcuda(g, e, "debug primitives");
}

void destroy_group(Group* g) {
    if (!g) return;
    for (int k = 0; k < 2; k++) {
        for (int c = 0; c < BC_NCOL; c++) cudaFree(g->bcol[k][c]);
        cudaFree(g->biiw[k]);
        for (int c = 0; c < CC_NCOL; c++) cudaFree(g->ccol[k][c]);
        g->cbuf[k].release();
    }
    cudaFree(g->bgrav); cudaFree(g->b_en); cudaFree(g->c_en); cudaFree(g->c_body); cudaFree(g->c_shape);
    cudaFree(g->c_leaf); cudaFreeHost(g->t_cleaf); cudaFree(g->d_tree_rows); cudaFree(g->d_fast);
    if (g->ev_step_copy) cudaEventDestroy(g->ev_step_copy);
    cudaFree(g->c_cat); cudaFree(g->c_mask); cudaFree(g->c_moved); cudaFree(g->pool); cudaFree(g->d_small);
    cudaFree(g->d_items); cudaFree(g->d_s1); cudaFree(g->d_s2); cudaFree(g->d_p1); cudaFree(g->d_r1);
    cudaFree(g->d_p2); cudaFree(g->d_r2); cudaFree(g->d_rep); cudaFree(g->d_coll); cudaFree(g->d_nct);
    cudaFree(g->d_cache); cudaFree(g->d_nd); cudaFree(g->d_l1); cudaFree(g->d_l2);
    cudaFree(g->d_mids); cudaFree(g->d_msrc); cudaFree(g->d_mprev); cudaFree(g->d_istart); cudaFree(g->d_icount);
    cudaFreeHost(g->h_items); cudaFreeHost(g->h_out); cudaFreeHost(g->h_mids); cudaFreeHost(g->h_msrc);
    cudaFreeHost(g->h_mprev); cudaFreeHost(g->h_istart); cudaFreeHost(g->h_icount); cudaFreeHost(g->h_step);
    cudaFreeHost(g->h_ijstart); cudaFreeHost(g->h_ijcount); cudaFreeHost(g->h_jlist);
    cudaFreeHost(g->h_reset);
    cudaFree(g->j_rec); cudaFree(g->d_jlist); cudaFree(g->d_ijstart); cudaFree(g->d_ijcount); cudaFree(g->d_jiisl);
    cudaFree(g->d_jibstart); cudaFree(g->d_jibcount); cudaFree(g->d_jirows);
    cudaFree(g->d_solver_stats);
    cudaFreeHost(g->h_hitems); cudaFreeHost(g->h_hrect); cudaFreeHost(g->h_hstart); cudaFreeHost(g->h_hpstart);
    cudaFreeHost(g->h_hprect); cudaFreeHost(g->h_hbatch); cudaFreeHost(g->h_hout);
    cudaFree(g->d_hitems); cudaFree(g->d_hrect); cudaFree(g->d_hstart); cudaFree(g->d_hpstart); cudaFree(g->d_hprect);
    cudaFree(g->d_hbatch); cudaFree(g->d_hout); cudaFree(g->d_hond); cudaFree(g->d_hol1); cudaFree(g->d_hol2);
    cudaFree(g->d_ts1); cudaFree(g->d_ts2); cudaFree(g->d_tp1); cudaFree(g->d_tr1); cudaFree(g->d_tp2);
    cudaFree(g->d_tr2); cudaFree(g->d_trep); cudaFree(g->d_tcoll); cudaFree(g->d_tnct); cudaFree(g->d_tmid);
    cudaFree(g->d_tnd); cudaFree(g->d_tl1); cudaFree(g->d_tl2); cudaFree(g->d_tri);
    cudaFree(g->d_tcache[0]); cudaFree(g->d_tcache[1]); cudaFree(g->d_hf);
    cudaFree(g->d_cm); cudaFree(g->d_ttri[0]); cudaFree(g->d_ttri[1]); cudaFree(g->d_herr); cudaFreeHost(g->h_herr);
    cudaFree(g->d_dbg_snap); cudaFree(g->d_dbg_lines); cudaFree(g->d_dbg_tris); cudaFree(g->d_dbg_jobs);
    cudaFree(g->d_dbg_points);
    if (g->tuner.e0) cudaEventDestroy(g->tuner.e0);
    if (g->tuner.e1) cudaEventDestroy(g->tuner.e1);
    cudaFreeHost(g->h_tnodes); cudaFree(g->d_tnodes); cudaFreeHost(g->h_tq); cudaFree(g->d_tq);
    cudaFreeHost(g->h_tleaves); cudaFree(g->d_tleaves); cudaFreeHost(g->h_tpos); cudaFree(g->d_tpos);
    cudaFreeHost(g->h_tcnt); cudaFree(g->d_tcnt);
    cudaFree(g->d_tree); cudaFree(g->d_tree_base); cudaFree(g->d_tree_hdr);
    cudaFreeHost(g->h_gq); cudaFree(g->d_gq);
    cudaFreeHost(g->h_rnodes); cudaFree(g->d_rnodes); cudaFreeHost(g->h_rcols); cudaFree(g->d_rcols);
    cudaFree(g->d_rhf); cudaFree(g->d_rays); cudaFree(g->d_rhits); cudaFree(g->d_rcount);
    if (g->ev_r0) cudaEventDestroy(g->ev_r0);
    if (g->ev_r1) cudaEventDestroy(g->ev_r1);
    if (g->ev_rect) cudaEventDestroy(g->ev_rect);
    cudaFreeHost(g->t_grav); cudaFreeHost(g->t_ben); cudaFreeHost(g->t_cen); cudaFreeHost(g->t_cbody);
    cudaFreeHost(g->t_cshape); cudaFreeHost(g->t_cat); cudaFreeHost(g->t_mask); cudaFreeHost(g->t_bperm);
    cudaFreeHost(g->t_cperm);
    delete g;
}

// Replays rp3dg_world_create's call sequence for one world on the host
// bookkeeping and fills that world's rows of the host columns.
int build_world(Group* g, WorldH& w, const rp3dg_body_desc* bd, uint32_t nb, const rp3dg_collider_desc* cd,
                uint32_t nc, std::vector<float4>* col, std::vector<float4>* ccols, std::vector<uint8_t>& dynamic,
                std::vector<int>& creation_order) {
    for (uint32_t i = 0; i < nc; i++) {
        if (cd[i].body < 0 || uint32_t(cd[i].body) >= nb || (i && cd[i].body < cd[i - 1].body))
            return cfail(g->ctx, RP3DG_EINVAL, "colliders must be grouped by body, bodies ascending");
        if (cd[i].shape < 0 || size_t(cd[i].shape) >= g->shapes.size())
            return cfail(g->ctx, RP3DG_EINVAL, "collider shape outside the shape table");
    }
    for (uint32_t i = 0; i < nb; i++)
        if (bd[i].type < RP3DG_BODY_STATIC || bd[i].type > RP3DG_BODY_DYNAMIC)
            return cfail(g->ctx, RP3DG_EINVAL, "bad body type");
    for (uint32_t i = 0; i < nc; i++)
        if (g->shapes[size_t(cd[i].shape)].kind == RP3DG_SHAPE_HEIGHTFIELD && bd[cd[i].body].type != RP3DG_BODY_STATIC)
            return cfail(g->ctx, RP3DG_EINVAL, "a height-field collider must belong to a static body");
    w.nb = nb;
    w.nc = nc;
    w.bodies.resize(nb);
    w.colliders.resize(nc);
    w.bcomp.reserve_ids(nb);
    w.ccomp.reserve_ids(nc);
    w.gravity.assign(nb, 1);
    w.body_debug.assign(nb, 0);
    dynamic.assign(nb, 0);
    for (int k = 0; k < BC_NCOL; k++) col[k].assign(nb, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int k = 0; k < CC_NCOL; k++) ccols[k].assign(nc, make_float4(0.f, 0.f, 0.f, 0.f));
    uint32_t ci = 0;
    for (uint32_t b = 0; b < nb; b++) {
        const rp3dg_body_desc& d = bd[b];
        BodyH& B = w.bodies[b];
        w.bcomp.add(int(b), false);  // createRigidBody: enabled, DYNAMIC
        col[BC_POS][b] = make_float4(d.position[0], d.position[1], d.position[2], 0.f);
        col[BC_ORI][b] = make_float4(d.orientation[0], d.orientation[1], d.orientation[2], d.orientation[3]);
        col[BC_MASS][b] = make_float4(1.0f, 1.0f, 0.0f, 0.0f);
        col[BC_IIL][b] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        col[BC_LLOCK][b] = make_float4(1.f, 1.f, 1.f, 0.f);
        col[BC_ALOCK][b] = make_float4(1.f, 1.f, 1.f, 0.f);
        std::vector<uint32_t> mine;
        while (ci < nc && uint32_t(cd[ci].body) == b) {
            const rp3dg_collider_desc& c = cd[ci];
            ColliderH& C = w.colliders[ci];
            C.body = int(b);
            C.shape = c.shape;
            const int kind = g->shapes[size_t(c.shape)].kind;
            C.convex = kind != RP3DG_SHAPE_HEIGHTFIELD && kind != RP3DG_SHAPE_CONCAVE_MESH;
            C.mesh = kind == RP3DG_SHAPE_CONCAVE_MESH;
            C.hf = C.convex ? -1 : g->shapes[size_t(c.shape)].mesh;
            C.category = c.category;
            C.mask = c.mask;
            // addCollider, then setIsTrigger(true): the collider stops being a
            // simulation collider and the body keeps one only if another
            // collider is (Collider.cpp:250-257, Body::updateHasSimulationCollider)
            C.trigger = (c.flags & RP3DG_COLLIDER_TRIGGER) != 0;
            w.ccomp.add(int(ci), !w.bcomp.enabled(int(b)));
            B.colliders.push_back(int(ci));
            if (!C.trigger) B.has_sim_collider = true;
            ccols[CC_LPOS][ci] = make_float4(c.position[0], c.position[1], c.position[2], 0.f);
            ccols[CC_LORI][ci] = make_float4(c.orientation[0], c.orientation[1], c.orientation[2], c.orientation[3]);
            // Material::mFrictionCoefficientSqrt = sqrt(friction)
            ccols[CC_MAT][ci] = make_float4(std::sqrt(c.friction), c.bounciness, 0.f, 0.f);
            creation_order.push_back(int(ci));
            mine.push_back(ci);
            ci++;
        }
        if (d.type == RP3DG_BODY_DYNAMIC) {
            // updateMassPropertiesFromColliders (RigidBody.cpp:548-608)
            float total = 0.0f, com[3] = {0.f, 0.f, 0.f};
            for (uint32_t k : mine) {
                float in[3], m;
                if (!shape_mass(g->ctx, g->shapes[size_t(cd[k].shape)], cd[k].mass_density, in, &m))
                    return cfail(g->ctx, RP3DG_EINVAL, "mass properties of a concave or unknown collider shape");
                total += m;
                for (int a = 0; a < 3; a++) com[a] += m * cd[k].position[a];
            }
            if (total > 0.0f)
                for (int a = 0; a < 3; a++) com[a] /= total;
            float tmp[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
            float total2 = 0.0f;
            for (uint32_t k : mine) {
                float in[3], m;
                shape_mass(g->ctx, g->shapes[size_t(cd[k].shape)], cd[k].mass_density, in, &m);
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
        w.gravity[b] = d.gravity_enabled ? 1 : 0;
        B.allowed_sleep = d.allowed_to_sleep != 0;
        if (d.type != RP3DG_BODY_STATIC) {
            col[BC_LV][b] = make_float4(d.linear_velocity[0], d.linear_velocity[1], d.linear_velocity[2], 0.f);
            col[BC_AV][b] = make_float4(d.angular_velocity[0], d.angular_velocity[1], d.angular_velocity[2], 0.f);
        }
    }
    w.dev_body_at = w.bcomp.at;
    w.dev_col_at = w.ccomp.at;
    return 0;
}

int ensure_manifold_staging(Group* g, uint32_t NM, uint32_t NI);

int create_group(rp3dg_ctx* ctx, const rp3dg_world_settings* s, uint32_t nworlds, const uint32_t* boff,
                 const rp3dg_body_desc* bd, const uint32_t* coff, const rp3dg_collider_desc* cd, int nthreads,
                 Group** out) {
    if (!ctx || !s || !out || !boff || !coff) return ctx ? cfail(ctx, RP3DG_EINVAL, "null argument") : RP3DG_EINVAL;
    *out = nullptr;
    auto* g = new Group();
    g->ctx = ctx;
    g->stream = static_cast<cudaStream_t>(rp3dg_stream(ctx));
    g->set = *s;
    g->nthreads = nthreads > 0 ? nthreads : 1;
    if (rp3dg::get_shapes_host(ctx, &g->shapes) || g->shapes.empty()) {
        destroy_group(g);
        return cfail(ctx, RP3DG_EINVAL, "no shape table (rp3dg_set_shapes)");
    }
    if (nworlds == 0) {
        destroy_group(g);
        return cfail(ctx, RP3DG_EINVAL, "no world");
    }
    // concave mesh instances of the context, by id, and the middle phase's error word
    {
        std::vector<rp3dg::CmDesc> cms;
        rp3dg::get_cmeshes(ctx, &cms);
        if ((!cms.empty() && (cudaMalloc(&g->d_cm, cms.size() * sizeof(rp3dg::CmDesc)) != cudaSuccess ||
                              cudaMemcpy(g->d_cm, cms.data(), cms.size() * sizeof(rp3dg::CmDesc),
                                         cudaMemcpyHostToDevice) != cudaSuccess)) ||
            cudaMalloc(&g->d_herr, 4) != cudaSuccess || cudaMemset(g->d_herr, 0, 4) != cudaSuccess ||
            cudaMallocHost(&g->h_herr, 4) != cudaSuccess) {
            destroy_group(g);
            return cfail(ctx, RP3DG_ENOMEM, "concave-mesh tables");
        }
        *g->h_herr = 0;
        g->n_cm = uint32_t(cms.size());
    }
    // height fields named by the shape table, by id
    {
        std::vector<rp3dg::HfDesc> hfs;
        for (const rp3dg_shape& sh : g->shapes) {
            if (sh.kind != RP3DG_SHAPE_HEIGHTFIELD) continue;
            if (size_t(sh.mesh) >= hfs.size()) hfs.resize(size_t(sh.mesh) + 1, rp3dg::HfDesc{});
            if (rp3dg::get_heightfield(ctx, sh.mesh, &hfs[size_t(sh.mesh)])) {
                destroy_group(g);
                return cfail(ctx, RP3DG_EINVAL, "shape refers to an unknown height field");
            }
        }
        if (!hfs.empty()) {
            g->n_hf = uint32_t(hfs.size());
            if (cudaMalloc(&g->d_hf, hfs.size() * sizeof(rp3dg::HfDesc)) != cudaSuccess ||
                cudaMemcpy(g->d_hf, hfs.data(), hfs.size() * sizeof(rp3dg::HfDesc), cudaMemcpyHostToDevice) != cudaSuccess) {
                destroy_group(g);
                return cfail(ctx, RP3DG_ENOMEM, "height-field tables");
            }
        }
    }
    // the event after the concave pairs' rectangles / mesh counts are read back
    if (cudaEventCreateWithFlags(&g->ev_rect, cudaEventDisableTiming) != cudaSuccess) {
        destroy_group(g);
        return cfail(ctx, RP3DG_ENOMEM, "middle-phase event");
    }
    g->worlds.resize(nworlds);
    std::vector<float4> col[BC_NCOL], ccols[CC_NCOL];
    std::vector<float4> wcol[BC_NCOL], wccols[CC_NCOL];
    std::vector<uint8_t> dyn_all, dyn;
    std::vector<std::vector<int>> orders(nworlds);
    uint32_t NB = 0, NC = 0;
    for (uint32_t k = 0; k < nworlds; k++) {
        if (boff[k + 1] < boff[k] || coff[k + 1] < coff[k]) {
            destroy_group(g);
            return cfail(ctx, RP3DG_EINVAL, "world offsets must not decrease");
        }
        WorldH& w = g->worlds[k];
        w.b0 = NB;
        w.c0 = NC;
        int rc = build_world(g, w, bd + boff[k], boff[k + 1] - boff[k], cd + coff[k], coff[k + 1] - coff[k], wcol,
                             wccols, dyn, orders[k]);
        if (rc) {
            destroy_group(g);
            return rc;
        }
        // host columns in component order
        for (int c = 0; c < BC_NCOL; c++)
            for (uint32_t r = 0; r < w.nb; r++) col[c].push_back(wcol[c][size_t(w.bcomp.at[r])]);
        for (uint32_t r = 0; r < w.nb; r++) dyn_all.push_back(dyn[size_t(w.bcomp.at[r])]);
        for (int c = 0; c < CC_NCOL; c++)
            for (uint32_t r = 0; r < w.nc; r++) ccols[c].push_back(wccols[c][size_t(w.ccomp.at[r])]);
        NB += w.nb;
        NC += w.nc;
    }
    g->NB = NB;
    g->NC = NC;
    cudaError_t e = cudaSuccess;
    auto M = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 16)); };
    for (int k = 0; k < 2; k++) {
        for (int c = 0; c < BC_NCOL; c++) M((void**)&g->bcol[k][c], size_t(NB) * 16);
        M((void**)&g->biiw[k], size_t(NB) * 48);
        for (int c = 0; c < CC_NCOL; c++) M((void**)&g->ccol[k][c], size_t(NC) * 16);
    }
    M((void**)&g->bgrav, NB); M((void**)&g->b_en, NB); M((void**)&g->c_en, NC);
    M((void**)&g->c_body, size_t(NC) * 4); M((void**)&g->c_shape, size_t(NC) * 4); M((void**)&g->c_leaf, size_t(NC) * 4);
    M((void**)&g->c_cat, size_t(NC) * 2); M((void**)&g->c_mask, size_t(NC) * 2); M((void**)&g->c_moved, NC);
    uint8_t* d_dyn = nullptr;
    M((void**)&d_dyn, NB);
    if (e != cudaSuccess) {
        cudaFree(d_dyn);
        destroy_group(g);
        return cfail(ctx, RP3DG_ENOMEM, "cudaMalloc(world)");
    }
    for (int c = 0; c < BC_NCOL; c++)
        if (NB) cudaMemcpyAsync(g->bcol[0][c], col[c].data(), size_t(NB) * 16, cudaMemcpyHostToDevice, g->stream);
    cudaMemsetAsync(g->biiw[0], 0, size_t(NB) * 48, g->stream);
    for (int c = 0; c < CC_NCOL; c++)
        if (NC) cudaMemcpyAsync(g->ccol[0][c], ccols[c].data(), size_t(NC) * 16, cudaMemcpyHostToDevice, g->stream);
    if (NB) cudaMemcpyAsync(d_dyn, dyn_all.data(), NB, cudaMemcpyHostToDevice, g->stream);
    g->tables_dirty = true;
    int rc = sync_rows(g);
    if (rc) {
        cudaFree(d_dyn);
        destroy_group(g);
        return rc;
    }
    const uint32_t n = std::max(NB, NC);
    if (n)
        world_setup<<<blocks(n), 128, 0, g->stream>>>(NB, g->bcol[0][BC_POS], g->bcol[0][BC_ORI], g->bcol[0][BC_COML],
                                                      g->bcol[0][BC_COMW], d_dyn, NC, g->c_body, g->ccol[0][CC_LPOS],
                                                      g->ccol[0][CC_LORI], g->ccol[0][CC_WPOS], g->ccol[0][CC_WORI]);
    // constrained position / orientation: the centre of mass and orientation
    // (setType(STATIC) sets them from the transform, RigidBody.cpp:80-82)
    if (NB) {
        cudaMemcpyAsync(g->bcol[0][BC_XC], g->bcol[0][BC_COMW], size_t(NB) * 16, cudaMemcpyDeviceToDevice, g->stream);
        cudaMemcpyAsync(g->bcol[0][BC_QC], g->bcol[0][BC_ORI], size_t(NB) * 16, cudaMemcpyDeviceToDevice, g->stream);
    }
    e = cudaStreamSynchronize(g->stream);
    cudaFree(d_dyn);
    if (e != cudaSuccess) {
        destroy_group(g);
        return cfail(ctx, RP3DG_ECUDA, "world set-up kernel");
    }
    for (uint32_t k = 0; k < nworlds; k++) {
        WorldH& w = g->worlds[k];
        const rp3dg_body_desc* d = bd + boff[k];
        w.init_pose.resize(w.nb);
        for (uint32_t b = 0; b < w.nb; b++) {
            w.init_pose[b].p[0] = d[b].position[0]; w.init_pose[b].p[1] = d[b].position[1]; w.init_pose[b].p[2] = d[b].position[2];
            for (int c = 0; c < 4; c++) w.init_pose[b].q[c] = d[b].orientation[c];
        }
    }
    // initial fat AABBs of every collider (addCollider -> addObject)
    if (NC) {
        uint8_t* force = nullptr;
        cudaMalloc(&force, NC);
        cudaMemsetAsync(force, 1, NC, g->stream);
        rp3dg_broadphase bp{};
        bp.n = NC;
        bp.n_update = NC;
        bp.shape = g->c_shape;
        bp.body = g->c_body;
        bp.world_position = reinterpret_cast<rp3dg_float4*>(g->ccol[0][CC_WPOS]);
        bp.world_orientation = reinterpret_cast<rp3dg_float4*>(g->ccol[0][CC_WORI]);
        bp.force_reinsert = force;
        bp.fat_min = reinterpret_cast<rp3dg_float4*>(g->ccol[0][CC_FMIN]);
        bp.fat_max = reinterpret_cast<rp3dg_float4*>(g->ccol[0][CC_FMAX]);
        bp.moved = g->c_moved;
        rc = rp3dg_broadphase_update_device(ctx, &bp);
        std::vector<float4> fmin(NC), fmax(NC);
        cudaMemcpyAsync(fmin.data(), g->ccol[0][CC_FMIN], size_t(NC) * 16, cudaMemcpyDeviceToHost, g->stream);
        cudaMemcpyAsync(fmax.data(), g->ccol[0][CC_FMAX], size_t(NC) * 16, cudaMemcpyDeviceToHost, g->stream);
        e = cudaStreamSynchronize(g->stream);
        cudaFree(force);
        if (rc || e != cudaSuccess) {
            destroy_group(g);
            return rc ? rc : cfail(ctx, RP3DG_ECUDA, "initial broad phase");
        }
        for (uint32_t k = 0; k < nworlds; k++) {
            WorldH& w = g->worlds[k];
            for (int c : orders[k]) {
                const uint32_t r = w.c0 + uint32_t(w.ccomp.slot[size_t(c)]);
                Box box;
                box.mn[0] = fmin[r].x; box.mn[1] = fmin[r].y; box.mn[2] = fmin[r].z;
                box.mx[0] = fmax[r].x; box.mx[1] = fmax[r].y; box.mx[2] = fmax[r].z;
                const int id = w.tree.add_object(box, c);
                w.colliders[size_t(c)].bp = id;
                if (size_t(id) >= w.bp_to_collider.size()) w.bp_to_collider.resize(size_t(id) + 1, -1);
                w.bp_to_collider[size_t(id)] = c;
                w.moved.add(id);
            }
            w.moved_at.assign(w.colliders.size(), 0);
            // the filter fields of each leaf's collider, side by side
            w.leaf_info.assign(w.bp_to_collider.size(), LeafInfo{});
            for (size_t id = 0; id < w.bp_to_collider.size(); id++) {
                const int c = w.bp_to_collider[id];
                if (c < 0) continue;
                const ColliderH& C = w.colliders[size_t(c)];
                w.leaf_info[id] = LeafInfo{C.body, C.category, C.mask};
            }
        }
        // the row tables now hold each collider's tree leaf at the next sync
        g->tables_dirty = true;
    }
    // the narrow phase's step buffers sized up front for twice as many convex
    // pairs as colliders (four times for a single world: a resting 100,000-
    // body world has ~3.5): growing them later frees and maps hundreds of MB
    // (16 contact slots per pair), which stalls the step that does it
    rc = ensure_items(g, (nworlds == 1 ? 4 : 2) * size_t(g->NC) + 1024);
    // and, for the same reason, the manifold staging, the island arrays and
    // both contact buffers for twice as many manifolds as colliders (two
    // points each: a resting 100,000-body world has ~1.25 manifolds and ~2
    // points per collider)
    if (!rc) rc = ensure_manifold_staging(g, g->NC, g->NC / 2 + 64);
    if (!rc) rc = ensure_pool(g, 2 * size_t(g->NC) + 1024);
    if (!rc && (g->cbuf[0].ensure(2 * g->NC + 64, 4 * g->NC + 64) || g->cbuf[1].ensure(2 * g->NC + 64, 4 * g->NC + 64)))
        rc = wfail(g, RP3DG_ENOMEM, "cudaMalloc(contacts)");
    // a group of small worlds keeps its trees on the device (one GPU thread
    // per world replays that world's reinsertions); one large world keeps its
    // tree on the host, whose sequential reinsertions are faster there
    if (!rc && nworlds >= 2) {
        size_t most = 0;
        for (const WorldH& w : g->worlds) most = std::max(most, w.colliders.size());
        if (most <= DEV_TREE_MAX_COLLIDERS) {
            rc = upload_trees(g);
            g->dev_tree = rc == 0;
        }
    }
    if (rc) {
        destroy_group(g);
        return rc;
    }
    *out = g;
    return 0;
}

// Manifold staging (ids, sources, previous manifolds) and island arrays of a
// step, grown to twice what is needed.
int ensure_manifold_staging(Group* g, uint32_t NM, uint32_t NI) {
    if (g->cap_hm < NM || !g->h_mids) {
        const size_t cap = std::max<size_t>(size_t(NM) * 2, 64);
        cudaFreeHost(g->h_mids); cudaFreeHost(g->h_msrc); cudaFreeHost(g->h_mprev);
        cudaFree(g->d_mids); cudaFree(g->d_msrc); cudaFree(g->d_mprev);
        g->h_mids = g->h_msrc = g->h_mprev = nullptr;
        g->d_mids = g->d_msrc = g->d_mprev = nullptr;
        g->cap_hm = 0;
        if (cudaMallocHost(&g->h_mids, cap * 16) || cudaMallocHost(&g->h_msrc, cap * 16) ||
            cudaMallocHost(&g->h_mprev, cap * 16) || cudaMalloc(&g->d_mids, cap * 16) ||
            cudaMalloc(&g->d_msrc, cap * 16) || cudaMalloc(&g->d_mprev, cap * 16))
            return wfail(g, RP3DG_ENOMEM, "allocation of manifold staging");
        g->cap_hm = cap;
    }
    if (g->cap_hi < NI || !g->h_istart) {
        const size_t cap = std::max<size_t>(size_t(NI) * 2, 64);
        cudaFreeHost(g->h_istart); cudaFreeHost(g->h_icount); cudaFree(g->d_istart); cudaFree(g->d_icount);
        cudaFreeHost(g->h_ijstart); cudaFreeHost(g->h_ijcount); cudaFree(g->d_ijstart); cudaFree(g->d_ijcount);
        g->h_istart = g->h_icount = g->h_ijstart = g->h_ijcount = nullptr;
        g->d_istart = g->d_icount = g->d_ijstart = g->d_ijcount = nullptr;
        g->cap_hi = 0;
        if (cudaMallocHost(&g->h_istart, cap * 4) || cudaMallocHost(&g->h_icount, cap * 4) ||
            cudaMalloc(&g->d_istart, cap * 4) || cudaMalloc(&g->d_icount, cap * 4) ||
            cudaMallocHost(&g->h_ijstart, cap * 4) || cudaMallocHost(&g->h_ijcount, cap * 4) ||
            cudaMalloc(&g->d_ijstart, cap * 4) || cudaMalloc(&g->d_ijcount, cap * 4))
            return wfail(g, RP3DG_ENOMEM, "allocation of island arrays");
        g->cap_hi = cap;
    }
    return 0;
}

void tuner_step(Group* g);

int update_group(Group* g, float dt) {
    if (!g) return RP3DG_EINVAL;
    if (!(dt > 0.0f)) return wfail(g, RP3DG_EINVAL, "dt must be positive");
    g->state_version++;
    cudaStream_t st = g->stream;
    rp3dg_ctx* ctx = g->ctx;
    std::memset(&g->stats, 0, sizeof(g->stats));
    // phase timer: with profiling on, the stream is drained at each mark so
    // that GPU time is charged to the phase that queued it
    auto mark = [&](int k) {
        if (!g->profiling) return;
        cudaStreamSynchronize(st);
        const auto now = std::chrono::steady_clock::now();
        g->phase_ms[k] += std::chrono::duration<double, std::milli>(now - g->t_mark).count();
        g->t_mark = now;
    };
    if (g->profiling) g->t_mark = std::chrono::steady_clock::now();

    // ---- broad phase and middle phase of every world (host order, GPU fat AABBs)
    if (g->dev_tree) {
        const int rq = tree_queries_group(g);
        if (rq) return rq;
    }
    for_worlds(g, [&](int k) { broad_and_middle_phase(g, g->worlds[size_t(k)]); });
    mark(0);
    if (g->profiling) {
        // broad-phase sub-phases summed over the worlds (13..15)
        for (WorldH& w : g->worlds)
            for (int q = 0; q < 3; q++) {
                g->phase_ms[13 + q] += w.prof_bp[q];
                w.prof_bp[q] = 0.0;
            }
    }
    // batches: algorithm-major, worlds in order inside a batch
    // sub-phase marks of phase 1 (8..12)
    auto sub = [&](int k) {
        if (!g->profiling) return;
        cudaStreamSynchronize(st);
        const auto now = std::chrono::steady_clock::now();
        g->phase_ms[k] += std::chrono::duration<double, std::milli>(now - g->t_mark).count();
        g->t_mark = now;
    };
    uint32_t T = 0;
    for (int a = 0; a < NB_ALGOS; a++) {
        g->batch_start[a] = T;
        for (WorldH& w : g->worlds) {
            w.item_off[a] = T - g->batch_start[a];
            T += uint32_t(w.items[a].size());
        }
    }
    g->batch_start[NB_ALGOS] = T;
    g->stats.narrowphase_tests = T;
    // convex vs concave pairs, laid out the same way
    uint32_t CI = 0;
    for (int a = 0; a < NB_ALGOS; a++) {
        g->hitem_start[a] = CI;
        for (WorldH& w : g->worlds) {
            w.hitem_off[a] = CI - g->hitem_start[a];
            CI += uint32_t(w.hitems[a].size());
        }
    }
    g->hitem_start[NB_ALGOS] = CI;
    int rc = ensure_pool(g);
    if (rc) return rc;
    sub(8);
    size_t nreset = 0;
    for (WorldH& w : g->worlds) nreset += w.reset_slots.size();
    if (nreset) {
        if (host_grow(&g->h_reset, &g->cap_hreset, nreset) || dev_grow(&g->d_small, &g->cap_small, nreset))
            return wfail(g, RP3DG_ENOMEM, "allocation of cache resets");
        size_t o = 0;
        for (WorldH& w : g->worlds) {
            std::memcpy(g->h_reset + o, w.reset_slots.data(), w.reset_slots.size() * 4);
            o += w.reset_slots.size();
            w.reset_slots.clear();
        }
        cudaMemcpyAsync(g->d_small, g->h_reset, nreset * 4, cudaMemcpyHostToDevice, st);
        world_reset_cache<<<blocks(uint32_t(nreset)), 128, 0, st>>>(uint32_t(nreset), g->d_small, g->pool);
    }
    sub(9);
    rc = sync_rows(g);
    if (rc) return rc;
    sub(10);
    if (T) {
        rc = ensure_items(g, T);
        if (rc) return rc;
    }
    sub(12);
    for_worlds(g, [&](int k) {
        WorldH& w = g->worlds[size_t(k)];
        for (int a = 0; a < NB_ALGOS; a++)
            if (!w.items[a].empty())
                std::memcpy(g->h_items + g->batch_start[a] + w.item_off[a], w.items[a].data(), w.items[a].size() * 16);
    });
    const int cc = g->cur_c;
    // ---- middle phase of the convex vs concave pairs: the cell rectangle of
    // each pair first (read back while the convex pairs' narrow phase runs)
    if (CI) {
        rc = ensure_hitems(g, CI);
        if (rc) return rc;
        for_worlds(g, [&](int k) {
            WorldH& w = g->worlds[size_t(k)];
            for (int a = 0; a < NB_ALGOS; a++)
                if (!w.hitems[a].empty())
                    std::memcpy(g->h_hitems + g->hitem_start[a] + w.hitem_off[a], w.hitems[a].data(),
                                w.hitems[a].size() * 16);
        });
        const rp3dg_shape* d_shapes = nullptr;
        const float4* d_bounds = nullptr;
        rp3dg::get_shape_device(ctx, &d_shapes, &d_bounds);
        cudaMemcpyAsync(g->d_hitems, g->h_hitems, size_t(CI) * 16, cudaMemcpyHostToDevice, st);
        HfRectArgs ra;
        ra.n = CI;
        ra.items = g->d_hitems;
        ra.c_shape = g->c_shape;
        ra.shapes = d_shapes;
        ra.bounds = d_bounds;
        ra.c_wpos = g->ccol[cc][CC_WPOS];
        ra.c_wori = g->ccol[cc][CC_WORI];
        ra.hf = g->d_hf;
        ra.cm = g->d_cm;
        ra.rect = g->d_hrect;
        ra.error = g->d_herr;
        cudaError_t e = launch_hf_rects(ra, st);
        if (e != cudaSuccess) return wcuda(g, e, "height-field middle phase");
        cudaMemcpyAsync(g->h_hrect, g->d_hrect, size_t(CI) * 16, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(g->h_herr, g->d_herr, 4, cudaMemcpyDeviceToHost, st);
        cudaEventRecord(g->ev_rect, st);
    }
    mark(1);
    if (T) {
        cudaMemcpyAsync(g->d_items, g->h_items, size_t(T) * 16, cudaMemcpyHostToDevice, st);
        GatherArgs ga;
        ga.n = T;
        ga.items = g->d_items;
        ga.c_shape = g->c_shape;
        ga.c_wpos = g->ccol[cc][CC_WPOS];
        ga.c_wori = g->ccol[cc][CC_WORI];
        ga.pool = g->pool;
        ga.s1 = g->d_s1; ga.s2 = g->d_s2;
        ga.p1 = g->d_p1; ga.r1 = g->d_r1; ga.p2 = g->d_p2; ga.r2 = g->d_r2;
        ga.report = g->d_rep;
        ga.cache = g->d_cache;
        world_gather_batch<<<blocks(T), 128, 0, st>>>(ga);
        // ---- narrow phase + manifold step, one call per algorithm batch
        for (int a = 0; a < NB_ALGOS; a++) {
            const uint32_t s0 = g->batch_start[a], n = g->batch_start[a + 1] - s0;
            if (!n) continue;
            rp3dg_pair_batch pb{};
            pb.n = n;
            pb.shape1 = g->d_s1 + s0; pb.shape2 = g->d_s2 + s0;
            pb.pos1 = reinterpret_cast<rp3dg_float4*>(g->d_p1 + s0);
            pb.rot1 = reinterpret_cast<rp3dg_float4*>(g->d_r1 + s0);
            pb.pos2 = reinterpret_cast<rp3dg_float4*>(g->d_p2 + s0);
            pb.rot2 = reinterpret_cast<rp3dg_float4*>(g->d_r2 + s0);
            pb.report_contacts = g->d_rep + s0;
            pb.cache = g->d_cache + s0;
            rp3dg_contact_batch cbt{};
            cbt.is_colliding = g->d_coll + s0;
            cbt.nb_contacts = g->d_nct + s0;
            cbt.normal_depth = reinterpret_cast<rp3dg_float4*>(g->d_nd + size_t(s0) * MAXC);
            cbt.local1 = reinterpret_cast<rp3dg_float4*>(g->d_l1 + size_t(s0) * MAXC);
            cbt.local2 = reinterpret_cast<rp3dg_float4*>(g->d_l2 + size_t(s0) * MAXC);
            cbt.max_contacts = MAXC;
            rc = rp3dg_narrowphase_device(ctx, a + 1, &pb, &cbt, 1);
            if (rc) return rc;
            rc = rp3dg_reduce_contacts_device(ctx, &pb, &cbt, nullptr);
            if (rc) return rc;
        }
        world_scatter_cache<<<blocks(T), 128, 0, st>>>(T, g->d_items, g->d_cache, g->pool);
        cudaMemcpyAsync(g->h_out, g->d_coll, T, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(g->h_out + T, g->d_nct, T, cudaMemcpyDeviceToHost, st);
    }
    // ---- triangle tests of the convex vs concave pairs and their manifolds
    if (CI) {
        cudaError_t e = cudaEventSynchronize(g->ev_rect);
        if (e != cudaSuccess) return wcuda(g, e, "height-field middle phase");
        if (*g->h_herr) return wfail(g, RP3DG_ECAPACITY, "concave mesh middle phase: tree deeper than the query stack");
        // HeightField::computeOverlappingTriangles: two triangles per cell of
        // [iMin, iMax) x [jMin, jMax); a concave mesh: the triangles its tree
        // query found; tests algorithm-major like the items
        uint32_t TC = 0;
        bool any_mesh = false;
        for (int a = 0; a < NB_ALGOS; a++) {
            g->htest_start[a] = TC;
            for (uint32_t ci = g->hitem_start[a]; ci < g->hitem_start[a + 1]; ci++) {
                const int4 r = g->h_hrect[ci];
                g->h_hstart[ci] = TC;
                if (g->h_hitems[ci].w & HF_MESH) {
                    any_mesh = true;
                    TC += uint32_t(r.y);
                } else if (r.y > r.x && r.w > r.z) {
                    TC += 2u * uint32_t(r.y - r.x) * uint32_t(r.w - r.z);
                }
            }
        }
        g->htest_start[NB_ALGOS] = TC;
        g->h_hstart[CI] = TC;
        g->stats.narrowphase_tests += TC;
        // per item: its batch, and the records of the step before (the pair
        // keeps them only if that step tested it)
        for (int a = 0; a < NB_ALGOS; a++) {
            const int4 batch = make_int4(int(g->htest_start[a]), int(g->htest_start[a + 1] - g->htest_start[a]), 0, 0);
            for (WorldH& w : g->worlds) {
                const uint32_t base = g->hitem_start[a] + w.hitem_off[a];
                for (uint32_t i = 0; i < w.hitems[a].size(); i++) {
                    const uint32_t ci = base + i;
                    PairH& p = w.concave[w.hitem_pair[a][i]];
                    g->h_hbatch[ci] = batch;
                    g->h_hpstart[ci] = p.rec_valid ? p.rec_start : -1;
                    g->h_hprect[ci] = p.rec_rect;
                    p.rec_valid = true;
                    p.rec_start = int(g->h_hstart[ci]);
                    p.rec_rect = g->h_hrect[ci];
                }
            }
        }
        rc = ensure_htests(g, TC);
        if (rc) return rc;
        cudaMemcpyAsync(g->d_hstart, g->h_hstart, size_t(CI + 1) * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->d_hbatch, g->h_hbatch, size_t(CI) * 16, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->d_hpstart, g->h_hpstart, size_t(CI) * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->d_hprect, g->h_hprect, size_t(CI) * 16, cudaMemcpyHostToDevice, st);
        const int cur = g->cur_tc;
        if (TC && any_mesh) {
            const rp3dg_shape* d_shapes = nullptr;
            const float4* d_bounds = nullptr;
            rp3dg::get_shape_device(ctx, &d_shapes, &d_bounds);
            HfListArgs la;
            la.n = CI;
            la.items = g->d_hitems;
            la.start = g->d_hstart;
            la.c_shape = g->c_shape;
            la.shapes = d_shapes;
            la.bounds = d_bounds;
            la.c_wpos = g->ccol[cc][CC_WPOS];
            la.c_wori = g->ccol[cc][CC_WORI];
            la.cm = g->d_cm;
            la.tri_id = g->d_ttri[cur];
            la.error = g->d_herr;
            e = launch_hf_list(la, st);
            if (e != cudaSuccess) return wcuda(g, e, "concave mesh triangles");
        }
        if (TC) {
            HfTestArgs ta;
            ta.n_items = CI;
            ta.n_tests = TC;
            ta.items = g->d_hitems;
            ta.rect = g->d_hrect;
            ta.start = g->d_hstart;
            ta.batch = g->d_hbatch;
            ta.prev_start = g->d_hpstart;
            ta.prev_rect = g->d_hprect;
            ta.c_shape = g->c_shape;
            ta.c_wpos = g->ccol[cc][CC_WPOS];
            ta.c_wori = g->ccol[cc][CC_WORI];
            ta.hf = g->d_hf;
            ta.cm = g->d_cm;
            ta.tri_id = g->d_ttri[cur];
            ta.prev_tri_id = g->d_ttri[1 - cur];
            ta.error = g->d_herr;
            ta.prev_cache = g->d_tcache[1 - cur];
            ta.s1 = g->d_ts1; ta.s2 = g->d_ts2;
            ta.p1 = g->d_tp1; ta.r1 = g->d_tr1; ta.p2 = g->d_tp2; ta.r2 = g->d_tr2;
            ta.report = g->d_trep;
            ta.cache = g->d_tcache[cur];
            ta.tri = g->d_tri;
            e = launch_hf_tests(ta, st);
            if (e != cudaSuccess) return wcuda(g, e, "height-field triangles");
            for (int a = 0; a < NB_ALGOS; a++) {
                const uint32_t s0 = g->htest_start[a], n = g->htest_start[a + 1] - s0;
                if (!n) continue;
                rp3dg_pair_batch pb{};
                pb.n = n;
                pb.shape1 = g->d_ts1 + s0; pb.shape2 = g->d_ts2 + s0;
                pb.pos1 = reinterpret_cast<rp3dg_float4*>(g->d_tp1 + s0);
                pb.rot1 = reinterpret_cast<rp3dg_float4*>(g->d_tr1 + s0);
                pb.pos2 = reinterpret_cast<rp3dg_float4*>(g->d_tp2 + s0);
                pb.rot2 = reinterpret_cast<rp3dg_float4*>(g->d_tr2 + s0);
                pb.report_contacts = g->d_trep + s0;
                pb.cache = g->d_tcache[cur] + s0;
                rp3dg_contact_batch cbt{};
                cbt.is_colliding = g->d_tcoll + s0;
                cbt.nb_contacts = g->d_tnct + s0;
                cbt.normal_depth = reinterpret_cast<rp3dg_float4*>(g->d_tnd + size_t(s0) * MAXC);
                cbt.local1 = reinterpret_cast<rp3dg_float4*>(g->d_tl1 + size_t(s0) * MAXC);
                cbt.local2 = reinterpret_cast<rp3dg_float4*>(g->d_tl2 + size_t(s0) * MAXC);
                cbt.max_contacts = MAXC;
                rc = rp3dg::narrowphase_tri_device(ctx, a + 1, &pb, &cbt, g->d_tri + rp3dg::TRI_REC * size_t(s0));
                if (rc) return rc;
            }
        }
        HfManifoldArgs ma;
        ma.n_items = CI;
        ma.items = g->d_hitems;
        ma.start = g->d_hstart;
        ma.batch = g->d_hbatch;
        ma.c_wori = g->ccol[cc][CC_WORI];
        ma.cos_similar = g->set.cos_angle_similar_contact_manifold;
        ma.is_colliding = g->d_tcoll;
        ma.nb_contacts = g->d_tnct;
        ma.nd = g->d_tnd; ma.l1 = g->d_tl1; ma.l2 = g->d_tl2;
        ma.cache = g->d_tcache[cur];
        ma.mid = g->d_tmid;
        // the uchar4 counts first: 4-byte aligned whatever CI is
        ma.out_npts = reinterpret_cast<uchar4*>(g->d_hout);
        ma.out_coll = g->d_hout + 4 * size_t(CI);
        ma.out_nman = g->d_hout + 5 * size_t(CI);
        ma.out_nd = g->d_hond; ma.out_l1 = g->d_hol1; ma.out_l2 = g->d_hol2;
        e = launch_hf_manifolds(ma, st);
        if (e != cudaSuccess) return wcuda(g, e, "concave manifolds");
        cudaMemcpyAsync(g->h_hout, g->d_hout, size_t(CI) * 6, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(g->h_herr, g->d_herr, 4, cudaMemcpyDeviceToHost, st);
    }
    g->cur_tc = 1 - g->cur_tc;
    if (T || CI) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return wcuda(g, e, "narrow phase");
        if (CI && *g->h_herr) return wfail(g, RP3DG_ECAPACITY, "concave mesh middle phase: inconsistent triangle lists");
    }
    mark(2);
    // ---- contact pairs and islands of every world
    const uint8_t* h_coll = g->h_out;
    const uint8_t* h_count = g->h_out + T;
    const uint8_t* h_hnpts = g->h_hout;
    const uint8_t* h_hcoll = g->h_hout + 4 * size_t(CI);
    const uint8_t* h_hnman = g->h_hout + 5 * size_t(CI);
    for_worlds(g, [&](int k) {
        contacts_and_islands(g, g->worlds[size_t(k)], h_coll, h_count, h_hcoll, h_hnman, h_hnpts);
    });
    uint32_t NM = 0, NP = 0, NI = 0;
    for (WorldH& w : g->worlds) {
        w.man_base = NM;
        w.pt_base = NP;
        w.isl_base = NI;
        NM += w.nm;
        NP += w.np;
        NI += uint32_t(w.islands.size());
        g->stats.contact_pairs += uint32_t(w.cpairs.size());
    }
    g->stats.manifolds = NM;
    g->stats.contact_points = NP;
    g->stats.islands = NI;
    rc = ensure_manifold_staging(g, NM, NI);
    if (rc) return rc;
    // joints of every world, back to back
    uint32_t NJ = 0;
    for (WorldH& w : g->worlds) {
        w.jl_base = NJ;
        NJ += uint32_t(w.jlist.size());
    }
    if (NJ && (host_grow(&g->h_jlist, &g->cap_hjl, NJ) || dev_grow(&g->d_jlist, &g->cap_jl, NJ)))
        return wfail(g, RP3DG_ENOMEM, "allocation of joint lists");
    mark(3);
    // rows may have moved (bodies woken by the islands): sync before packing ids
    rc = sync_rows(g);
    if (rc) return rc;
    for_worlds(g, [&](int k) { fill_manifolds(g, g->worlds[size_t(k)]); });
    const int bc = g->cur_b, ccur = g->cur_c;
    // islands with joints and their enabled bodies' rows (for the position correction)
    std::vector<uint32_t> ji_island, ji_bstart, ji_bcount;
    std::vector<int32_t> ji_rows;
    if (NJ) {
        // the worlds' lists (fill_manifolds) back to back
        size_t nisl = 0, nrows = 0;
        for (WorldH& w : g->worlds) {
            w.ji_off = uint32_t(nisl);
            w.ji_row_off = uint32_t(nrows);
            nisl += w.ji_isl.size();
            nrows += w.ji_rows.size();
        }
        ji_island.resize(nisl);
        ji_bstart.resize(nisl);
        ji_bcount.resize(nisl);
        ji_rows.resize(nrows);
        for_worlds(g, [&](int k) {
            const WorldH& w = g->worlds[size_t(k)];
            uint32_t r = w.ji_row_off;
            for (size_t i = 0; i < w.ji_isl.size(); i++) {
                ji_island[w.ji_off + i] = w.ji_isl[i];
                ji_bstart[w.ji_off + i] = r;
                ji_bcount[w.ji_off + i] = w.ji_bcount[i];
                r += w.ji_bcount[i];
            }
            if (!w.ji_rows.empty())
                std::memcpy(ji_rows.data() + w.ji_row_off, w.ji_rows.data(), w.ji_rows.size() * 4);
        });
        if (dev_grow(&g->d_jiisl, &g->cap_ji, ji_island.size() + 1) ||
            dev_grow(&g->d_jibstart, &g->cap_jbs, ji_island.size() + 1) ||
            dev_grow(&g->d_jibcount, &g->cap_jbc, ji_island.size() + 1) ||
            dev_grow(&g->d_jirows, &g->cap_jr, ji_rows.size() + 1))
            return wfail(g, RP3DG_ENOMEM, "allocation of joint islands");
        cudaMemcpyAsync(g->d_jlist, g->h_jlist, size_t(NJ) * 16, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->d_ijstart, g->h_ijstart, size_t(NI) * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->d_ijcount, g->h_ijcount, size_t(NI) * 4, cudaMemcpyHostToDevice, st);
        if (!ji_island.empty()) {
            cudaMemcpyAsync(g->d_jiisl, ji_island.data(), ji_island.size() * 4, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(g->d_jibstart, ji_bstart.data(), ji_bstart.size() * 4, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(g->d_jibcount, ji_bcount.data(), ji_bcount.size() * 4, cudaMemcpyHostToDevice, st);
        }
        if (!ji_rows.empty())
            cudaMemcpyAsync(g->d_jirows, ji_rows.data(), ji_rows.size() * 4, cudaMemcpyHostToDevice, st);
    }
    ContactBuf& CB = g->cbuf[g->cur_cb];
    ContactBuf& PB = g->cbuf[1 - g->cur_cb];
    if (CB.ensure(std::max<uint32_t>(NM, 1), std::max<uint32_t>(NP, 1))) return wfail(g, RP3DG_ENOMEM, "cudaMalloc(contacts)");
    if (NM) {
        cudaMemcpyAsync(g->d_mids, g->h_mids, size_t(NM) * 16, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->d_msrc, g->h_msrc, size_t(NM) * 16, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->d_mprev, g->h_mprev, size_t(NM) * 16, cudaMemcpyHostToDevice, st);
        PackArgs a;
        a.nm = NM;
        a.ids = g->d_mids;
        a.src = g->d_msrc;
        a.prev = g->d_mprev;
        a.kept_count = g->d_nct;
        a.b_nd = g->d_nd; a.b_l1 = g->d_l1; a.b_l2 = g->d_l2;
        a.c_nd = g->d_hond; a.c_l1 = g->d_hol1; a.c_l2 = g->d_hol2;
        a.cos_similar = g->set.cos_angle_similar_contact_manifold;
        a.persist2 = g->set.persistent_contact_distance_threshold * g->set.persistent_contact_distance_threshold;
        a.pm_pstart = PB.pstart; a.pm_fv1 = PB.fv1; a.pm_fv2 = PB.fv2; a.pm_fimp = PB.fimp;
        a.pp_nd = PB.nd; a.pp_l1 = PB.l1; a.pp_imp = PB.imp; a.pp_rest = PB.rest;
        a.m_ids = CB.ids; a.m_pstart = CB.pstart; a.m_npts = CB.npts;
        a.m_fv1 = CB.fv1; a.m_fv2 = CB.fv2; a.m_fimp = CB.fimp;
        a.p_nd = CB.nd; a.p_l1 = CB.l1; a.p_l2 = CB.l2; a.p_imp = CB.imp; a.p_rest = CB.rest;
        world_pack_contacts<<<blocks(NM), 128, 0, st>>>(a);
    }
    CB.nm = NM;
    CB.np = NP;
    if (NI) {
        cudaMemcpyAsync(g->d_istart, g->h_istart, size_t(NI) * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(g->d_icount, g->h_icount, size_t(NI) * 4, cudaMemcpyHostToDevice, st);
    }
    mark(4);
    // DebugRenderer::onContact runs before the integration: keep the
    // collider transforms it reads
    if ((g->debug_items & (RP3DG_DEBUG_CONTACT_POINT | RP3DG_DEBUG_CONTACT_NORMAL)) && g->NC) {
        if (dev_grow(&g->d_dbg_snap, &g->cap_dbg_snap, 2 * size_t(g->NC)))
            return wfail(g, RP3DG_ENOMEM, "cudaMalloc(debug snapshot)");
        cudaMemcpyAsync(g->d_dbg_snap, g->ccol[ccur][CC_WPOS], size_t(g->NC) * 16, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(g->d_dbg_snap + g->NC, g->ccol[ccur][CC_WORI], size_t(g->NC) * 16, cudaMemcpyDeviceToDevice,
                        st);
    }
    // ---- dynamics stage (inertia, velocities, solver, positions, state)
    {
        rp3dg_dynamics_params pr{};
        pr.dt = dt;
        pr.gravity[0] = g->set.gravity[0]; pr.gravity[1] = g->set.gravity[1]; pr.gravity[2] = g->set.gravity[2];
        pr.gravity_enabled = 1;
        pr.velocity_iterations = g->set.velocity_iterations;
        pr.split_impulse = 1;
        pr.restitution_velocity_threshold = g->set.restitution_velocity_threshold;
        auto F = [](float4* p) { return reinterpret_cast<rp3dg_float4*>(p); };
        rp3dg_bodies B{};
        B.n = g->NB;
        B.n_enabled = 0;  // per-row flags
        B.position = F(g->bcol[bc][BC_POS]); B.orientation = F(g->bcol[bc][BC_ORI]);
        B.com_world = F(g->bcol[bc][BC_COMW]); B.com_local = F(g->bcol[bc][BC_COML]);
        B.linear_velocity = F(g->bcol[bc][BC_LV]); B.angular_velocity = F(g->bcol[bc][BC_AV]);
        B.force = F(g->bcol[bc][BC_F]); B.torque = F(g->bcol[bc][BC_T]);
        B.inv_inertia_local = F(g->bcol[bc][BC_IIL]); B.inv_inertia_world = F(g->biiw[bc]);
        B.mass = F(g->bcol[bc][BC_MASS]); B.linear_lock = F(g->bcol[bc][BC_LLOCK]); B.angular_lock = F(g->bcol[bc][BC_ALOCK]);
        B.gravity = g->bgrav;
        rp3dg_colliders C{};
        C.n = g->NC;
        C.n_enabled = 0;
        C.body = g->c_body;
        C.local_position = F(g->ccol[ccur][CC_LPOS]); C.local_orientation = F(g->ccol[ccur][CC_LORI]);
        C.world_position = F(g->ccol[ccur][CC_WPOS]); C.world_orientation = F(g->ccol[ccur][CC_WORI]);
        C.material = F(g->ccol[ccur][CC_MAT]);
        rp3dg_manifolds Mf{};
        Mf.n = NM;
        Mf.ids = reinterpret_cast<int32_t*>(CB.ids);
        Mf.point_start = CB.pstart; Mf.nb_points = CB.npts;
        Mf.friction_vector1 = F(CB.fv1); Mf.friction_vector2 = F(CB.fv2); Mf.friction_impulse = F(CB.fimp);
        rp3dg_points P{};
        P.n = NP;
        P.normal_depth = F(CB.nd); P.local1 = F(CB.l1); P.local2 = F(CB.l2);
        P.penetration_impulse = CB.imp; P.is_resting = CB.rest;
        rp3dg_islands I{};
        I.n = NI;
        I.manifold_start = g->d_istart;
        I.manifold_count = g->d_icount;
        rp3dg::DynJoints J{};
        if (NJ) {
            J.nj = NJ;
            J.j_list = g->d_jlist;
            J.j_rec = g->j_rec;
            J.i_jstart = g->d_ijstart;
            J.i_jcount = g->d_ijcount;
            J.nji = uint32_t(ji_island.size());
            J.ji_island = g->d_jiisl;
            J.ji_bstart = g->d_jibstart;
            J.ji_bcount = g->d_jibcount;
            J.ji_rows = g->d_jirows;
            J.xc = g->bcol[bc][BC_XC];
            J.qc = g->bcol[bc][BC_QC];
            J.position_iterations = g->set.position_iterations;
        }
        // the candidate of this step while the autotuner runs
        Group::Tuner& tu = g->tuner;
        const bool tuning = tu.active && !tu.cands.empty();
        const rp3dg::DynTuning tn = tuning ? tu.cands[size_t(tu.idx) % tu.cands.size()] : g->tune;
        if (tuning) cudaEventRecord(tu.e0, st);
        rp3dg::DynSolver sol;
        sol.colored = g->solver;
        sol.stats = g->solver_stats ? g->d_solver_stats : nullptr;
        rc = rp3dg::dynamics_step_flags(ctx, &pr, &B, &C, &Mf, &P, &I, g->b_en, g->c_en, NJ ? &J : nullptr, &tn,
                                        &sol);
        if (rc) return rc;
        if (tuning) {
            cudaEventRecord(tu.e1, st);
            tu.timed = true;
            tu.nm = NM;
        }
        // the pageable joint-island vectors are read by the copies above
        if (NJ) cudaStreamSynchronize(st);
    }
    mark(5);
    // ---- updateColliders: world AABBs, fat-AABB test, reinsertion flags
    const size_t step_bytes = ((size_t(g->NC) + 15) & ~size_t(15)) + size_t(g->NC) * 32 + size_t(g->NB) + 64;
    if (host_grow(&g->h_step, &g->cap_hstep, step_bytes)) return wfail(g, RP3DG_ENOMEM, "cudaMallocHost(step)");
    uint8_t* h_moved = g->h_step;
    float4* h_fmin = reinterpret_cast<float4*>(g->h_step + ((size_t(g->NC) + 15) & ~size_t(15)));
    float4* h_fmax = h_fmin + g->NC;
    uint8_t* h_fast = reinterpret_cast<uint8_t*>(h_fmax + g->NC);
    if (g->NC) {
        rp3dg_broadphase bp{};
        bp.n = g->NC;
        bp.n_update = g->NC;
        bp.shape = g->c_shape;
        bp.body = g->c_body;
        bp.world_position = reinterpret_cast<rp3dg_float4*>(g->ccol[ccur][CC_WPOS]);
        bp.world_orientation = reinterpret_cast<rp3dg_float4*>(g->ccol[ccur][CC_WORI]);
        bp.fat_min = reinterpret_cast<rp3dg_float4*>(g->ccol[ccur][CC_FMIN]);
        bp.fat_max = reinterpret_cast<rp3dg_float4*>(g->ccol[ccur][CC_FMAX]);
        bp.moved = g->c_moved;
        rc = rp3dg::broadphase_update_flags(ctx, &bp, g->c_en);
        if (rc) return rc;
        cudaMemcpyAsync(h_moved, g->c_moved, g->NC, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(h_fmin, g->ccol[ccur][CC_FMIN], size_t(g->NC) * 16, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(h_fmax, g->ccol[ccur][CC_FMAX], size_t(g->NC) * 16, cudaMemcpyDeviceToHost, st);
    }
    if (g->set.sleeping_enabled && g->NB) {
        if (dev_grow(&g->d_fast, &g->cap_fast, g->NB)) return wfail(g, RP3DG_ENOMEM, "cudaMalloc(sleep test)");
        world_sleep_fast<<<blocks(g->NB), 128, 0, st>>>(
            g->NB, g->bcol[bc][BC_LV], g->bcol[bc][BC_AV], g->set.sleep_linear_velocity * g->set.sleep_linear_velocity,
            g->set.sleep_angular_velocity * g->set.sleep_angular_velocity, g->d_fast);
        cudaMemcpyAsync(h_fast, g->d_fast, g->NB, cudaMemcpyDeviceToHost, st);
    }
    cudaError_t e;
    if (g->dev_tree && g->NC) {
        // the device trees' reinsertions run while the host does the sleep
        // bookkeeping below (the next step's queries wait for them)
        cudaEventRecord(g->ev_step_copy, st);
        rc = reinsert_on_device(g, g->c_moved, g->ccol[ccur][CC_FMIN], g->ccol[ccur][CC_FMAX]);
        if (rc) return rc;
        e = cudaEventSynchronize(g->ev_step_copy);
    } else {
        e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return wcuda(g, e, "step");
    mark(6);
    // ---- reinsertions and sleeping of every world
    for_worlds(g, [&](int k) { colliders_and_sleep(g, g->worlds[size_t(k)], dt, h_moved, h_fmin, h_fmax, h_fast); });
    // velocities / forces of bodies put to sleep (rows in the current device order)
    std::vector<int32_t> rows;
    for (WorldH& w : g->worlds) {
        if (w.slept.empty()) continue;
        std::vector<int32_t> row_of(w.nb);
        for (uint32_t r = 0; r < w.nb; r++) row_of[size_t(w.dev_body_at[r])] = int32_t(w.b0 + r);
        for (int b : w.slept)
            if (w.bodies[size_t(b)].sleeping) rows.push_back(row_of[size_t(b)]);
    }
    if (!rows.empty()) {
        if (ensure_small(g, rows.size())) return RP3DG_ENOMEM;
        cudaMemcpyAsync(g->d_small, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, st);
        world_zero_rows<<<blocks(uint32_t(rows.size())), 128, 0, st>>>(uint32_t(rows.size()), g->d_small,
                                                                       g->bcol[bc][BC_LV], g->bcol[bc][BC_AV],
                                                                       g->bcol[bc][BC_F], g->bcol[bc][BC_T]);
    }
    // resetBodiesForceAndTorque
    cudaMemsetAsync(g->bcol[bc][BC_F], 0, size_t(g->NB) * 16, st);
    cudaMemsetAsync(g->bcol[bc][BC_T], 0, size_t(g->NB) * 16, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return wcuda(g, e, "end of step");
    tuner_step(g);
    g->cur_cb = 1 - g->cur_cb;
    rc = debug_primitives(g);
    if (rc) return rc;
    for (WorldH& w : g->worlds) {
        w.stepped = true;
        g->stats.overlapping_pairs += uint32_t(w.pairs.size() + w.concave.size());
        g->stats.disabled_pairs += w.stats.disabled_pairs;
        g->stats.enabled_bodies += w.stats.enabled_bodies;
        g->stats.moved_colliders += w.stats.moved_colliders;
    }
    mark(7);
    return 0;
}

// The candidates of one autotuner phase: the current scheduling with one
// parameter varied (0: thread-per-island limit, 1: one-CTA-per-island
// threshold, 2: warp-kernel CTAs per SM).
std::vector<rp3dg::DynTuning> tuner_candidates(const rp3dg::DynTuning& base, int phase) {
    std::vector<rp3dg::DynTuning> c;
    const uint32_t small[] = {4, 8, 16, 32}, giant[] = {128, 256, 512}, per_sm[] = {1, 2};
    if (phase == 0) for (uint32_t v : small) { rp3dg::DynTuning t = base; t.small_max = v; c.push_back(t); }
    if (phase == 1) for (uint32_t v : giant) { rp3dg::DynTuning t = base; t.giant_min = v; c.push_back(t); }
    if (phase == 2) for (uint32_t v : per_sm) { rp3dg::DynTuning t = base; t.large_per_sm = v; c.push_back(t); }
    return c;
}

// After a step's end: record the timed candidate; at the end of a phase keep
// the candidate with the lowest median time per manifold and start the next.
void tuner_step(Group* g) {
    Group::Tuner& tu = g->tuner;
    if (!tu.active || !tu.timed) return;
    tu.timed = false;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, tu.e0, tu.e1) != cudaSuccess) return;
    const size_t k = size_t(tu.idx) % tu.cands.size();
    tu.score[k].push_back(ms / float(std::max<uint32_t>(tu.nm, 1)));
    tu.idx++;
    if (size_t(tu.idx) < tu.cands.size() * size_t(tu.rounds)) return;
    size_t best = 0;
    float best_t = 3.4e38f;
    for (size_t i = 0; i < tu.cands.size(); i++) {
        std::vector<float> v = tu.score[i];
        std::sort(v.begin(), v.end());
        const float med = v.empty() ? 3.4e38f : v[v.size() / 2];
        if (med < best_t) { best_t = med; best = i; }
    }
    g->tune = tu.cands[best];
    tu.phase++;
    tu.idx = 0;
    tu.cands = tuner_candidates(g->tune, tu.phase);
    tu.score.assign(tu.cands.size(), std::vector<float>());
    if (tu.cands.empty()) tu.active = false;
}

// Host quaternion / vector arithmetic with the reference's expression trees
// (Quaternion.h:349-378, Vector3.h:219-227), for the joints' local frames.
struct HQ { float x, y, z, w; };
HQ hq_mul(HQ a, HQ b) {
    return {a.w * b.x + b.w * a.x + a.y * b.z - a.z * b.y, a.w * b.y + b.w * a.y + a.z * b.x - a.x * b.z,
            a.w * b.z + b.w * a.z + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
void hq_rot(HQ q, const float* p, float* out) {
    const float prodX = q.w * p[0] + q.y * p[2] - q.z * p[1];
    const float prodY = q.w * p[1] + q.z * p[0] - q.x * p[2];
    const float prodZ = q.w * p[2] + q.x * p[1] - q.y * p[0];
    const float prodW = -q.x * p[0] - q.y * p[1] - q.z * p[2];
    out[0] = q.w * prodX - prodY * q.z + prodZ * q.y - prodW * q.x;
    out[1] = q.w * prodY - prodZ * q.x + prodX * q.z - prodW * q.y;
    out[2] = q.w * prodZ - prodX * q.y + prodY * q.x - prodW * q.z;
}
void hv_normalize(float* v) {
    const float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l < 1.1920928955078125e-07f) return;
    v[0] /= l; v[1] /= l; v[2] /= l;
}
// transform.getInverse() * point (Transform.h:162-195)
void inv_apply(const float* p, HQ q, const float* point, float* out) {
    const HQ iq{-q.x, -q.y, -q.z, q.w};
    const float np[3] = {-p[0], -p[1], -p[2]};
    float t[3], r[3];
    hq_rot(iq, np, t);
    hq_rot(iq, point, r);
    out[0] = r[0] + t[0]; out[1] = r[1] + t[1]; out[2] = r[2] + t[2];
}

int add_joints(Group* g, uint32_t world, const rp3dg_joint_desc* jd, uint32_t n) {
    if (world >= g->worlds.size() || (n && !jd)) return wfail(g, RP3DG_EINVAL, "bad joint arguments");
    WorldH& w = g->worlds[world];
    if (w.stepped) return wfail(g, RP3DG_EINVAL, "joints must be added before the first update");
    if (!w.joints.empty()) return wfail(g, RP3DG_EINVAL, "joints of a world are added in one call");
    if (world + 1 < g->worlds.size())
        for (uint32_t k = world + 1; k < g->worlds.size(); k++)
            if (!g->worlds[k].joints.empty()) return wfail(g, RP3DG_EINVAL, "add the joints of the worlds in order");
    for (uint32_t i = 0; i < n; i++) {
        const rp3dg_joint_desc& d = jd[i];
        if (d.type != RP3DG_JOINT_BALL_AND_SOCKET && d.type != RP3DG_JOINT_HINGE && d.type != RP3DG_JOINT_FIXED &&
            d.type != RP3DG_JOINT_SLIDER)
            return wfail(g, RP3DG_EINVAL, "bad joint type");
        if (d.body1 < 0 || d.body2 < 0 || uint32_t(d.body1) >= w.nb || uint32_t(d.body2) >= w.nb || d.body1 == d.body2)
            return wfail(g, RP3DG_EINVAL, "bad joint bodies");
    }
    std::vector<rp3dg::JointRec> recs(n);
    w.jbase = g->nj_total;
    w.joints.resize(n);
    w.jcomp.reserve_ids(n);
    w.bscomp.reserve_ids(n);
    w.fcomp.reserve_ids(n);
    w.hcomp.reserve_ids(n);
    w.scomp.reserve_ids(n);
    for (uint32_t j = 0; j < n; j++) {
        const rp3dg_joint_desc& d = jd[j];
        JointH& J = w.joints[j];
        J.type = d.type;
        J.b1 = d.body1;
        J.b2 = d.body2;
        J.motor_speed = d.motor_speed;
        const bool dis = !w.bcomp.enabled(J.b1) && !w.bcomp.enabled(J.b2);
        joint_type_comps(w, d.type).add(int(j), dis);
        w.jcomp.add(int(j), dis);
        if (!d.collision_enabled) w.nocollide[body_pair_key(J.b1, J.b2)] = 1;
        w.bodies[size_t(J.b1)].joints.push_back(int(j));
        w.bodies[size_t(J.b2)].joints.push_back(int(j));
        const auto& P1 = w.init_pose[size_t(J.b1)];
        const auto& P2 = w.init_pose[size_t(J.b2)];
        const HQ q1{P1.q[0], P1.q[1], P1.q[2], P1.q[3]}, q2{P2.q[0], P2.q[1], P2.q[2], P2.q[3]};
        float la1[3], la2[3];
        inv_apply(P1.p, q1, d.anchor, la1);
        inv_apply(P2.p, q2, d.anchor, la2);
        float4* q = recs[j].q;
        for (int r = 0; r < rp3dg::JR_ROWS; r++) q[r] = make_float4(0.f, 0.f, 0.f, 0.f);
        int flags = 0;
        if (d.type == RP3DG_JOINT_BALL_AND_SOCKET && d.cone_limit_enabled) flags |= rp3dg::JF_CONE;
        const bool limited = d.type == RP3DG_JOINT_HINGE || d.type == RP3DG_JOINT_SLIDER;
        if (limited && d.limit_enabled) flags |= rp3dg::JF_LIMIT;
        if (limited && d.motor_enabled) flags |= rp3dg::JF_MOTOR;
        q[rp3dg::JR_HDR] = make_float4(__int_as_float_host(d.type), __int_as_float_host(flags), 0.f, 0.f);
        q[rp3dg::JR_LA1] = make_float4(la1[0], la1[1], la1[2], 0.f);
        q[rp3dg::JR_LA2] = make_float4(la2[0], la2[1], la2[2], 0.f);
        if (d.type == RP3DG_JOINT_HINGE) {
            float ax1[3], ax2[3];
            hq_rot(HQ{-q1.x, -q1.y, -q1.z, q1.w}, d.axis, ax1);
            hq_rot(HQ{-q2.x, -q2.y, -q2.z, q2.w}, d.axis, ax2);
            hv_normalize(ax1);
            hv_normalize(ax2);
            HQ qd = hq_mul(q2, HQ{-q1.x, -q1.y, -q1.z, q1.w});
            const float l = std::sqrt(qd.x * qd.x + qd.y * qd.y + qd.z * qd.z + qd.w * qd.w);
            qd = HQ{qd.x / l, qd.y / l, qd.z / l, qd.w / l};
            q[rp3dg::JR_AX1] = make_float4(ax1[0], ax1[1], ax1[2], 0.f);
            q[rp3dg::JR_AX2] = make_float4(ax2[0], ax2[1], ax2[2], 0.f);
            q[rp3dg::JR_QINV] = make_float4(-qd.x, -qd.y, -qd.z, qd.w);
            q[rp3dg::JR_PARAM] = make_float4(0.f, d.min_angle, d.max_angle, d.motor_speed);
            q[rp3dg::JR_PARAM2] = make_float4(d.max_motor_torque, 0.f, 0.f, 0.f);
        } else if (d.type == RP3DG_JOINT_BALL_AND_SOCKET) {
            q[rp3dg::JR_PARAM] = make_float4(d.cone_limit_enabled ? d.cone_half_angle : float(3.141592653589), 0.f, 0.f, 0.f);
        } else {
            // FixedJoint / SliderJoint constructors (FixedJoint.cpp:35-58,
            // SliderJoint.cpp:37-72): inverse initial orientation difference
            // q2^-1 * q1, and the slider axis in body 1's frame, normalised
            const HQ qd = hq_mul(HQ{-q2.x, -q2.y, -q2.z, q2.w}, q1);
            q[rp3dg::JR_QINV] = make_float4(qd.x, qd.y, qd.z, qd.w);
            if (d.type == RP3DG_JOINT_SLIDER) {
                float ax1[3];
                hq_rot(HQ{-q1.x, -q1.y, -q1.z, q1.w}, d.axis, ax1);
                hv_normalize(ax1);
                q[rp3dg::JR_AX1] = make_float4(ax1[0], ax1[1], ax1[2], 0.f);
                q[rp3dg::JR_PARAM] = make_float4(0.f, d.min_angle, d.max_angle, d.motor_speed);
                q[rp3dg::JR_PARAM2] = make_float4(d.max_motor_torque, 0.f, 0.f, 0.f);
            }
        }
    }
    // records: the group's array grows (existing records copied)
    const size_t need = size_t(g->nj_total) + n;
    if (need > g->cap_jrec) {
        rp3dg::JointRec* nr = nullptr;
        const size_t cap = std::max<size_t>(need, g->cap_jrec * 2);
        if (cudaMalloc(&nr, cap * sizeof(rp3dg::JointRec)) != cudaSuccess)
            return wfail(g, RP3DG_ENOMEM, "cudaMalloc(joint records)");
        if (g->nj_total)
            cudaMemcpyAsync(nr, g->j_rec, size_t(g->nj_total) * sizeof(rp3dg::JointRec), cudaMemcpyDeviceToDevice, g->stream);
        cudaStreamSynchronize(g->stream);
        cudaFree(g->j_rec);
        g->j_rec = nr;
        g->cap_jrec = cap;
    }
    if (n)
        cudaMemcpyAsync(g->j_rec + g->nj_total, recs.data(), size_t(n) * sizeof(rp3dg::JointRec), cudaMemcpyHostToDevice,
                        g->stream);
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return wcuda(g, e, "joint records");
    g->nj_total += n;
    return 0;
}

int read_bodies(Group* g, uint32_t world, bool all, float* position, float* orientation, float* linear_velocity,
                float* angular_velocity, uint8_t* sleeping) {
    const uint32_t n = g->NB;
    std::vector<float4> p(n), q(n), lv(n), av(n);
    const int b = g->cur_b;
    cudaMemcpyAsync(p.data(), g->bcol[b][BC_POS], size_t(n) * 16, cudaMemcpyDeviceToHost, g->stream);
    cudaMemcpyAsync(q.data(), g->bcol[b][BC_ORI], size_t(n) * 16, cudaMemcpyDeviceToHost, g->stream);
    cudaMemcpyAsync(lv.data(), g->bcol[b][BC_LV], size_t(n) * 16, cudaMemcpyDeviceToHost, g->stream);
    cudaMemcpyAsync(av.data(), g->bcol[b][BC_AV], size_t(n) * 16, cudaMemcpyDeviceToHost, g->stream);
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return wcuda(g, e, "read bodies");
    uint32_t out_base = 0;
    for (uint32_t k = 0; k < g->worlds.size(); k++) {
        const WorldH& w = g->worlds[k];
        if (!all && k != world) continue;
        for (uint32_t r = 0; r < w.nb; r++) {
            const size_t id = out_base + size_t(w.dev_body_at[r]);
            const uint32_t row = w.b0 + r;
            if (position) { position[3 * id] = p[row].x; position[3 * id + 1] = p[row].y; position[3 * id + 2] = p[row].z; }
            if (orientation) {
                orientation[4 * id] = q[row].x; orientation[4 * id + 1] = q[row].y;
                orientation[4 * id + 2] = q[row].z; orientation[4 * id + 3] = q[row].w;
            }
            if (linear_velocity) {
                linear_velocity[3 * id] = lv[row].x; linear_velocity[3 * id + 1] = lv[row].y; linear_velocity[3 * id + 2] = lv[row].z;
            }
            if (angular_velocity) {
                angular_velocity[3 * id] = av[row].x; angular_velocity[3 * id + 1] = av[row].y; angular_velocity[3 * id + 2] = av[row].z;
            }
            if (sleeping) sleeping[id] = w.bodies[size_t(w.dev_body_at[r])].sleeping ? 1 : 0;
        }
        if (all) out_base += w.nb;
    }
    return 0;
}

}  // namespace

extern "C" {

int rp3dg_world_create(rp3dg_ctx* ctx, const rp3dg_world_settings* s, const rp3dg_body_desc* bd, uint32_t nb,
                       const rp3dg_collider_desc* cd, uint32_t nc, rp3dg_world** out) {
    if ((nb && !bd) || (nc && !cd)) return ctx ? cfail(ctx, RP3DG_EINVAL, "null argument") : RP3DG_EINVAL;
    const uint32_t boff[2] = {0, nb}, coff[2] = {0, nc};
    return create_group(ctx, s, 1, boff, bd, coff, cd, 1, out);
}

int rp3dg_world_group_create(rp3dg_ctx* ctx, const rp3dg_world_settings* s, uint32_t nb_worlds,
                             const uint32_t* body_offsets, const rp3dg_body_desc* bodies,
                             const uint32_t* collider_offsets, const rp3dg_collider_desc* colliders, int nb_threads,
                             rp3dg_world** out) {
    if (nb_worlds && (!bodies || !colliders)) return ctx ? cfail(ctx, RP3DG_EINVAL, "null argument") : RP3DG_EINVAL;
    return create_group(ctx, s, nb_worlds, body_offsets, bodies, collider_offsets, colliders, nb_threads, out);
}

void rp3dg_world_destroy(rp3dg_world* w) { destroy_group(w); }

int rp3dg_world_add_joints(rp3dg_world* w, const rp3dg_joint_desc* joints, uint32_t n) {
    if (!w) return RP3DG_EINVAL;
    return add_joints(w, 0, joints, n);
}

int rp3dg_world_group_add_joints(rp3dg_world* w, uint32_t world, const rp3dg_joint_desc* joints, uint32_t n) {
    if (!w) return RP3DG_EINVAL;
    return add_joints(w, world, joints, n);
}

// HingeJoint::setMotorSpeed / SliderJoint::setMotorSpeed (HingeJoint.cpp:168-177,
// SliderJoint.cpp:210-219): a new speed is stored and wakes the joint's two
// bodies (Joint::awakeBodies, Joint.cpp:74-86).
int rp3dg_world_set_motor_speed(rp3dg_world* g, uint32_t world, uint32_t joint, float speed) {
    if (!g) return RP3DG_EINVAL;
    if (world >= g->worlds.size() || joint >= g->worlds[world].joints.size())
        return wfail(g, RP3DG_EINVAL, "bad world or joint index");
    WorldH& w = g->worlds[world];
    JointH& J = w.joints[joint];
    if (J.type != RP3DG_JOINT_HINGE && J.type != RP3DG_JOINT_SLIDER)
        return wfail(g, RP3DG_EINVAL, "only hinge and slider joints have a motor");
    if (speed == J.motor_speed) return 0;
    J.motor_speed = speed;
    float4* row = g->j_rec[w.jbase + joint].q + rp3dg::JR_PARAM;
    cudaError_t e = cudaMemcpyAsync(reinterpret_cast<char*>(row) + 3 * sizeof(float), &J.motor_speed, sizeof(float),
                                    cudaMemcpyHostToDevice, g->stream);
    if (e != cudaSuccess) return wcuda(g, e, "motor speed");
    set_sleeping(g, w, J.b1, false);
    set_sleeping(g, w, J.b2, false);
    g->state_version++;
    return sync_rows(g);
}

// The ray kernel's view of world `world`: the broad-phase tree's nodes
// (children, fat AABBs, leaves as collider indices) and per collider its
// transform row, body, shape and category bits; rebuilt when the state
// changed since the last build.
int ray_tables(Group* g, uint32_t world) {
    if (g->ray_version == g->state_version && g->ray_world == world && g->d_rnodes) return 0;
    int rc = sync_rows(g);
    if (!rc) rc = download_tree(g, world);
    if (rc) return rc;
    WorldH& w = g->worlds[world];
    const size_t nn = std::max<size_t>(w.tree.nodes.size(), 1);
    const size_t nc = std::max<size_t>(w.colliders.size(), 1);
    if (!pair_grow(&g->h_rnodes, &g->d_rnodes, &g->cap_rnodes, nn) ||
        !pair_grow(&g->h_rcols, &g->d_rcols, &g->cap_rcols, nc))
        return wfail(g, RP3DG_ENOMEM, "allocation of raycast tables");
    for (size_t k = 0; k < w.tree.nodes.size(); k++) {
        const rp3dg::order::Tree::Node& N = w.tree.nodes[k];
        rp3dg::RayNode& R = g->h_rnodes[k];
        const bool leaf = N.height == 0;
        const int c0 = leaf ? -2 - N.data : N.child[0];
        const int c1 = leaf ? -1 : N.child[1];
        R.lo = make_float4(N.box.mn[0], N.box.mn[1], N.box.mn[2], __int_as_float_host(c0));
        R.hi = make_float4(N.box.mx[0], N.box.mx[1], N.box.mx[2], __int_as_float_host(c1));
    }
    for (size_t c = 0; c < w.colliders.size(); c++) {
        const ColliderH& C = w.colliders[c];
        g->h_rcols[c] = make_int4(int(w.c0) + w.ccomp.slot[c], C.body, C.shape, int(C.category));
    }
    std::vector<rp3dg::HfDesc> hf;
    rp3dg::get_heightfields(g->ctx, &hf);
    if (!hf.empty() && dev_grow(&g->d_rhf, &g->cap_rhf, hf.size()))
        return wfail(g, RP3DG_ENOMEM, "allocation of raycast tables");
    cudaStream_t st = g->stream;
    cudaMemcpyAsync(g->d_rnodes, g->h_rnodes, w.tree.nodes.size() * sizeof(rp3dg::RayNode), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(g->d_rcols, g->h_rcols, w.colliders.size() * sizeof(int4), cudaMemcpyHostToDevice, st);
    if (!hf.empty())
        cudaMemcpyAsync(g->d_rhf, hf.data(), hf.size() * sizeof(rp3dg::HfDesc), cudaMemcpyHostToDevice, st);
    g->nb_rhf = uint32_t(hf.size());
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return wcuda(g, e, "raycast tables");
    g->ray_version = g->state_version;
    g->ray_world = world;
    return 0;
}

// Rays, hits and counts in device memory (on the world's stream).
int raycast_device(Group* g, uint32_t world, const rp3dg_ray* rays, uint32_t n, int32_t mode, uint32_t max_hits,
                   rp3dg_raycast_hit* hits, uint32_t* nb_hits, float* kernel_ms) {
    int rc = ray_tables(g, world);
    if (rc) return rc;
    if (dev_grow(&g->d_rcount, &g->cap_rcount, 1))
        return wfail(g, RP3DG_ENOMEM, "allocation of the raycast error word");
    if (!g->ev_r0 && (cudaEventCreate(&g->ev_r0) != cudaSuccess || cudaEventCreate(&g->ev_r1) != cudaSuccess))
        return wfail(g, RP3DG_ECUDA, "cudaEventCreate(raycast)");
    cudaStream_t st = g->stream;
    WorldH& w = g->worlds[world];
    rp3dg::RayArgs a{};
    a.nodes = g->d_rnodes;
    a.root = w.tree.root;
    a.colliders = g->d_rcols;
    a.c_wpos = g->ccol[g->cur_c][CC_WPOS];
    a.c_wori = g->ccol[g->cur_c][CC_WORI];
    const float4* bounds = nullptr;
    rp3dg::get_shape_device(g->ctx, &a.shapes, &bounds);
    rp3dg::get_mesh_arena_device(g->ctx, &a.mesh_words);
    a.hfields = g->d_rhf;
    a.nb_hfields = g->nb_rhf;
    a.cmeshes = g->d_cm;
    a.nb_cmeshes = g->n_cm;
    a.rays = rays;
    a.n = n;
    a.mode = mode;
    a.max_hits = max_hits;
    a.hits = hits;
    a.nb_hits = nb_hits;
    a.error = g->d_rcount;
    cudaMemsetAsync(g->d_rcount, 0, sizeof(uint32_t), st);
    cudaEventRecord(g->ev_r0, st);
    cudaError_t e = rp3dg::launch_world_raycast(a, st);
    cudaEventRecord(g->ev_r1, st);
    if (e != cudaSuccess) return wcuda(g, e, "raycast kernel");
    uint32_t err = 0;
    cudaMemcpyAsync(&err, g->d_rcount, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return wcuda(g, e, "raycast");
    if (kernel_ms) cudaEventElapsedTime(kernel_ms, g->ev_r0, g->ev_r1);
    if (err & 1u) return wfail(g, RP3DG_ECAPACITY, "raycast: tree deeper than the traversal stack");
    return 0;
}

int raycast_args(Group* g, uint32_t world, const void* rays, uint32_t n, int32_t mode, uint32_t max_hits,
                 const void* hits, const void* nb_hits) {
    if (!g) return RP3DG_EINVAL;
    if (world >= g->worlds.size()) return wfail(g, RP3DG_EINVAL, "bad world index");
    if (mode != RP3DG_RAYCAST_CLOSEST && mode != RP3DG_RAYCAST_ANY && mode != RP3DG_RAYCAST_ALL)
        return wfail(g, RP3DG_EINVAL, "bad raycast mode");
    if (n && (!rays || !nb_hits || (max_hits && !hits))) return wfail(g, RP3DG_EINVAL, "null raycast array");
    return 0;
}

int rp3dg_world_raycast_device(rp3dg_world* g, uint32_t world, const rp3dg_ray* rays, uint32_t n, int32_t mode,
                               uint32_t max_hits, rp3dg_raycast_hit* hits, uint32_t* nb_hits, float* kernel_ms) {
    int rc = raycast_args(g, world, rays, n, mode, max_hits, hits, nb_hits);
    if (rc || n == 0) return rc;
    return raycast_device(g, world, rays, n, mode, max_hits, hits, nb_hits, kernel_ms);
}

int rp3dg_world_raycast(rp3dg_world* g, uint32_t world, const rp3dg_ray* rays, uint32_t n, int32_t mode,
                        uint32_t max_hits, rp3dg_raycast_hit* hits, uint32_t* nb_hits) {
    int rc = raycast_args(g, world, rays, n, mode, max_hits, hits, nb_hits);
    if (rc || n == 0) return rc;
    const size_t nh = size_t(n) * max_hits;
    if (dev_grow(&g->d_rays, &g->cap_rays, n) || dev_grow(&g->d_rhits, &g->cap_rhits, std::max<size_t>(nh, 1)) ||
        dev_grow(&g->d_rcount, &g->cap_rcount, size_t(n) + 1))
        return wfail(g, RP3DG_ENOMEM, "allocation of raycast buffers");
    cudaStream_t st = g->stream;
    cudaMemcpyAsync(g->d_rays, rays, size_t(n) * sizeof(rp3dg_ray), cudaMemcpyHostToDevice, st);
    // the error word sits after the counts
    uint32_t* counts = g->d_rcount + 1;
    rc = raycast_device(g, world, g->d_rays, n, mode, max_hits, g->d_rhits, counts, nullptr);
    if (rc) return rc;
    if (nh) cudaMemcpyAsync(hits, g->d_rhits, nh * sizeof(rp3dg_raycast_hit), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(nb_hits, counts, size_t(n) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return wcuda(g, e, "raycast results");
    return 0;
}

int rp3dg_world_update(rp3dg_world* w, float dt) { return update_group(w, dt); }

int rp3dg_world_get_bodies(rp3dg_world* w, float* position, float* orientation, float* linear_velocity,
                           float* angular_velocity, uint8_t* sleeping) {
    if (!w) return RP3DG_EINVAL;
    return read_bodies(w, 0, true, position, orientation, linear_velocity, angular_velocity, sleeping);
}

int rp3dg_world_group_get_bodies(rp3dg_world* w, uint32_t world, float* position, float* orientation,
                                 float* linear_velocity, float* angular_velocity, uint8_t* sleeping) {
    if (!w || world >= w->worlds.size()) return RP3DG_EINVAL;
    return read_bodies(w, world, false, position, orientation, linear_velocity, angular_velocity, sleeping);
}

int rp3dg_world_group_get_pairs(rp3dg_world* g, uint32_t world, uint64_t* ids, uint32_t capacity, uint32_t* n) {
    if (!g || !n || world >= g->worlds.size()) return RP3DG_EINVAL;
    const WorldH& w = g->worlds[world];
    uint32_t k = 0;
    for (const auto& p : w.pairs) { if (ids && k < capacity) ids[k] = p.id; k++; }
    for (const auto& p : w.disabled) { if (ids && k < capacity) ids[k] = p.id; k++; }
    for (const auto& p : w.concave) { if (ids && k < capacity) ids[k] = p.id; k++; }
    for (const auto& p : w.concave_dis) { if (ids && k < capacity) ids[k] = p.id; k++; }
    *n = k;
    return 0;
}

int rp3dg_world_get_pairs(rp3dg_world* w, uint64_t* ids, uint32_t capacity, uint32_t* n) {
    return rp3dg_world_group_get_pairs(w, 0, ids, capacity, n);
}

int rp3dg_world_group_get_contacts(rp3dg_world* g, uint32_t world, int32_t* body1, int32_t* body2, uint8_t* nb_points,
                                   uint32_t capacity, float* normal_depth, float* local1, float* local2,
                                   uint32_t capacity_points, uint32_t* nb_manifolds, uint32_t* nb_contact_points) {
    if (!g || world >= g->worlds.size()) return RP3DG_EINVAL;
    // the arrays of the last step are the "previous" buffer after the swap
    const ContactBuf& B = g->cbuf[1 - g->cur_cb];
    const WorldH& w = g->worlds[world];
    const std::vector<ContactPairH>& cps = w.prev_cpairs;
    if (nb_manifolds) *nb_manifolds = w.nm;
    if (nb_contact_points) *nb_contact_points = w.np;
    // manifold -> (contact pair, manifold of the pair): a convex vs concave
    // pair owns up to four consecutive manifolds
    std::vector<std::pair<uint32_t, uint32_t>> order(w.nm, std::make_pair(0u, 0u));
    for (uint32_t i = 0; i < cps.size(); i++)
        if (cps[i].in_island)
            for (uint32_t q = 0; q < cps[i].nman; q++) order[cps[i].manifold - w.man_base + q] = std::make_pair(i, q);
    for (uint32_t m = 0; m < w.nm && m < capacity; m++) {
        const ContactPairH& c = cps[order[m].first];
        if (body1) body1[m] = c.b1;
        if (body2) body2[m] = c.b2;
        if (nb_points) nb_points[m] = uint8_t(c.concave ? (c.npts >> (8 * order[m].second)) & 0xffu : c.k);
    }
    const uint32_t np = std::min(w.np, capacity_points);
    if (np) {
        if (normal_depth) cudaMemcpyAsync(normal_depth, B.nd + w.pt_base, size_t(np) * 16, cudaMemcpyDeviceToHost, g->stream);
        if (local1) cudaMemcpyAsync(local1, B.l1 + w.pt_base, size_t(np) * 16, cudaMemcpyDeviceToHost, g->stream);
        if (local2) cudaMemcpyAsync(local2, B.l2 + w.pt_base, size_t(np) * 16, cudaMemcpyDeviceToHost, g->stream);
    }
    cudaError_t e = cudaStreamSynchronize(g->stream);
    return e == cudaSuccess ? 0 : wcuda(g, e, "read contacts");
}

int rp3dg_world_get_contact_events(rp3dg_world* g, uint32_t world, rp3dg_contact_event* events, uint32_t capacity,
                                   float* normal_depth, float* local1, float* local2, uint32_t capacity_points,
                                   uint32_t* nb_events, uint32_t* nb_points) {
    if (!g || world >= g->worlds.size() || (capacity && !events)) return RP3DG_EINVAL;
    const ContactBuf& B = g->cbuf[1 - g->cur_cb];
    const WorldH& w = g->worlds[world];
    const std::vector<ContactPairH>& cps = w.prev_cpairs;
    // CollisionCallback::CallbackData keeps the pairs that are not triggers
    uint32_t ne = 0, np = 0;
    for (const ContactPairH& c : cps)
        if (!c.trigger) {
            ne++;
            if (c.in_island) np += c.k;
        }
    for (const ContactPairH& c : w.lost) ne += c.trigger ? 0u : 1u;
    if (nb_events) *nb_events = ne;
    if (nb_points) *nb_points = np;
    // the step's packed points of this world, then gathered pair by pair
    std::vector<float4> nd, l1, l2;
    const bool want = capacity_points && (normal_depth || local1 || local2) && w.np;
    if (want) {
        nd.resize(w.np);
        l1.resize(w.np);
        l2.resize(w.np);
        cudaMemcpyAsync(nd.data(), B.nd + w.pt_base, size_t(w.np) * 16, cudaMemcpyDeviceToHost, g->stream);
        cudaMemcpyAsync(l1.data(), B.l1 + w.pt_base, size_t(w.np) * 16, cudaMemcpyDeviceToHost, g->stream);
        cudaMemcpyAsync(l2.data(), B.l2 + w.pt_base, size_t(w.np) * 16, cudaMemcpyDeviceToHost, g->stream);
        cudaError_t e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) return wcuda(g, e, "read contact events");
    }
    uint32_t k = 0, pt = 0;
    auto emit = [&](const ContactPairH& c, int type, bool points) {
        const uint32_t n = points ? c.k : 0u;
        if (k < capacity) {
            rp3dg_contact_event& ev = events[k];
            ev.body1 = c.b1;
            ev.body2 = c.b2;
            ev.collider1 = c.c1;
            ev.collider2 = c.c2;
            ev.type = type;
            ev.first_point = pt;
            ev.nb_points = n;
        }
        for (uint32_t i = 0; i < n; i++, pt++) {
            if (!want || pt >= capacity_points) continue;
            const uint32_t src = c.point - w.pt_base + i;
            if (normal_depth) std::memcpy(normal_depth + 4 * size_t(pt), &nd[src], 16);
            if (local1) std::memcpy(local1 + 4 * size_t(pt), &l1[src], 16);
            if (local2) std::memcpy(local2 + 4 * size_t(pt), &l2[src], 16);
        }
        k++;
    };
    for (const ContactPairH& c : cps)
        if (!c.trigger) emit(c, c.prev ? RP3DG_CONTACT_STAY : RP3DG_CONTACT_START, c.in_island);
    for (const ContactPairH& c : w.lost)
        if (!c.trigger) emit(c, RP3DG_CONTACT_EXIT, false);
    return 0;
}

int rp3dg_world_get_trigger_events(rp3dg_world* g, uint32_t world, rp3dg_contact_event* events, uint32_t capacity,
                                   uint32_t* nb_events) {
    if (!g || world >= g->worlds.size() || (capacity && !events)) return RP3DG_EINVAL;
    const WorldH& w = g->worlds[world];
    uint32_t k = 0;
    auto emit = [&](const ContactPairH& c, int type) {
        if (k < capacity) {
            rp3dg_contact_event& ev = events[k];
            ev.body1 = c.b1;
            ev.body2 = c.b2;
            ev.collider1 = c.c1;
            ev.collider2 = c.c2;
            ev.type = type;
            ev.first_point = 0;
            ev.nb_points = 0;
        }
        k++;
    };
    // OverlapCallback::CallbackData with onlyReportTriggers: the trigger
    // contact pairs, then the lost trigger pairs
    for (const ContactPairH& c : w.prev_cpairs)
        if (c.trigger) emit(c, c.prev ? RP3DG_CONTACT_STAY : RP3DG_CONTACT_START);
    for (const ContactPairH& c : w.lost)
        if (c.trigger) emit(c, RP3DG_CONTACT_EXIT);
    if (nb_events) *nb_events = k;
    return 0;
}

int rp3dg_world_set_debug_rendering(rp3dg_world* g, uint32_t items) {
    if (!g || (items & ~0x3fu)) return RP3DG_EINVAL;
    // disabled, the renderer is no longer reset: the last primitives stay
    g->debug_items = items;
    return 0;
}

int rp3dg_world_set_body_debug(rp3dg_world* g, uint32_t world, int32_t body, int enabled) {
    if (!g || world >= g->worlds.size()) return RP3DG_EINVAL;
    WorldH& w = g->worlds[world];
    if (body >= int32_t(w.nb)) return RP3DG_EINVAL;
    if (body < 0) std::fill(w.body_debug.begin(), w.body_debug.end(), uint8_t(enabled ? 1 : 0));
    else w.body_debug[size_t(body)] = enabled ? 1 : 0;
    return 0;
}

int rp3dg_world_get_debug_primitives(rp3dg_world* g, uint32_t world, rp3dg_debug_line* lines, uint32_t cap_lines,
                                     rp3dg_debug_triangle* tris, uint32_t cap_tris, uint32_t* nb_lines,
                                     uint32_t* nb_tris, int device) {
    if (!g || world >= g->worlds.size() || (cap_lines && !lines) || (cap_tris && !tris)) return RP3DG_EINVAL;
    const WorldH& w = g->worlds[world];
    if (nb_lines) *nb_lines = w.dbg_nl;
    if (nb_tris) *nb_tris = w.dbg_nt;
    const uint32_t nl = std::min(w.dbg_nl, cap_lines), nt = std::min(w.dbg_nt, cap_tris);
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (nl) cudaMemcpyAsync(lines, g->d_dbg_lines + w.dbg_line0, size_t(nl) * sizeof(rp3dg_debug_line), kind, g->stream);
    if (nt) cudaMemcpyAsync(tris, g->d_dbg_tris + w.dbg_tri0, size_t(nt) * sizeof(rp3dg_debug_triangle), kind, g->stream);
    cudaError_t e = cudaStreamSynchronize(g->stream);
    return e == cudaSuccess ? 0 : wcuda(g, e, "read debug primitives");
}

int rp3dg_world_get_contacts(rp3dg_world* w, int32_t* body1, int32_t* body2, uint8_t* nb_points, uint32_t capacity,
                             float* normal_depth, float* local1, float* local2, uint32_t capacity_points,
                             uint32_t* nb_manifolds, uint32_t* nb_contact_points) {
    return rp3dg_world_group_get_contacts(w, 0, body1, body2, nb_points, capacity, normal_depth, local1, local2,
                                          capacity_points, nb_manifolds, nb_contact_points);
}

int rp3dg_world_get_stats(rp3dg_world* w, rp3dg_world_stats* s) {
    if (!w || !s) return RP3DG_EINVAL;
    *s = w->stats;
    return 0;
}

int rp3dg_world_autotune(rp3dg_world* w, int rounds) {
    if (!w || rounds < 1) return RP3DG_EINVAL;
    Group::Tuner& tu = w->tuner;
    if (!tu.e0 && (cudaEventCreate(&tu.e0) != cudaSuccess || cudaEventCreate(&tu.e1) != cudaSuccess))
        return wfail(w, RP3DG_ECUDA, "cudaEventCreate(autotuner)");
    tu.active = true;
    tu.rounds = rounds;
    tu.phase = 0;
    tu.idx = 0;
    tu.timed = false;
    tu.cands = tuner_candidates(w->tune, 0);
    tu.score.assign(tu.cands.size(), std::vector<float>());
    return 0;
}

int rp3dg_world_get_tuning(rp3dg_world* w, uint32_t* out) {
    if (!w || !out) return RP3DG_EINVAL;
    out[0] = w->tune.small_max;
    out[1] = w->tune.giant_min;
    out[2] = w->tune.large_per_sm;
    out[3] = w->tuner.active ? 1u : 0u;
    return 0;
}

int rp3dg_world_set_device_trees(rp3dg_world* g, int enable) {
    if (!g) return RP3DG_EINVAL;
    if (bool(enable) == g->dev_tree) return 0;
    if (enable) {
        const int rc = upload_trees(g);
        if (rc) return rc;
        g->dev_tree = true;
        return 0;
    }
    for (uint32_t k = 0; k < uint32_t(g->worlds.size()); k++) {
        const int rc = download_tree(g, k);
        if (rc) return rc;
    }
    g->dev_tree = false;
    return 0;
}

int rp3dg_world_get_device_trees(rp3dg_world* g, int* enabled) {
    if (!g || !enabled) return RP3DG_EINVAL;
    *enabled = g->dev_tree ? 1 : 0;
    return 0;
}

int rp3dg_world_set_threads(rp3dg_world* w, int threads) {
    if (!w || threads < 1) return RP3DG_EINVAL;
    w->nthreads = threads;
    return 0;
}

int rp3dg_world_set_solver(rp3dg_world* w, int solver, int stats) {
    if (!w || (solver != RP3DG_SOLVER_EXACT && solver != RP3DG_SOLVER_GRAPH_COLORED)) return RP3DG_EINVAL;
    if (stats && !w->d_solver_stats) {
        if (cudaMalloc(&w->d_solver_stats, sizeof(rp3dg::SolverStats)) != cudaSuccess) {
            w->d_solver_stats = nullptr;
            return wfail(w, RP3DG_ENOMEM, "cudaMalloc(solver statistics)");
        }
        cudaMemset(w->d_solver_stats, 0, sizeof(rp3dg::SolverStats));
    }
    w->solver = solver;
    w->solver_stats = stats != 0;
    return 0;
}

int rp3dg_world_get_solver_stats(rp3dg_world* w, rp3dg_solver_stats* out) {
    if (!w || !out) return RP3DG_EINVAL;
    std::memset(out, 0, sizeof(*out));
    if (!w->d_solver_stats) return 0;
    rp3dg::SolverStats st;
    cudaError_t e = cudaMemcpyAsync(&st, w->d_solver_stats, sizeof(st), cudaMemcpyDeviceToHost, w->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return wfail(w, RP3DG_ECUDA, "solver statistics");
    float mx;
    std::memcpy(&mx, &st.residual_max_bits, 4);
    out->residual_rms = st.points ? std::sqrt(st.residual_sq_sum / double(st.points)) : 0.0;
    out->residual_max = mx;
    out->kinetic_energy = st.kinetic;
    out->potential_energy = st.potential;
    out->contact_points = st.points;
    out->colors = st.colors;
    out->coloring_rounds = st.rounds;
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
    for (uint32_t i = 0; i < n && i < 16; i++) ms[i] = w->phase_ms[i];
    return 0;
}

}  // extern "C"
