// Narrow-phase kernels: one launch per algorithm batch, one pair per thread.
// Pair inputs are struct-of-arrays (float4 transforms, int32 shape indices),
// outputs are slot-major so consecutive pairs write consecutive addresses.
// Convex-mesh tables (half-edges, faces, normals, vertices) are staged in
// shared memory once per CTA; the box topology comes from constant memory.
#include <cuda_runtime.h>

#include "axis_mlp.cuh"
#include "narrowphase.cuh"
#include "np_launch.h"

// Kernel tuning knobs (compile time): resident CTAs per SM requested from the
// register allocator, for the closed-form/GJK kernels, the warp-per-pair
// polyhedron kernels (one per shape combination, each with one SAT
// instantiation: 5 CTAs of 96 registers without spills, 7% faster on the
// hull-box batch than 4 CTAs) and the thread-per-pair polyhedron kernel
// (box-box only: 103 registers at 4 CTAs; at 5 it spills and is slower).
#ifndef RP3DG_NP_MIN_BLOCKS
#define RP3DG_NP_MIN_BLOCKS 4
#endif
#ifndef RP3DG_NP_MIN_BLOCKS_POLY_WARP
#define RP3DG_NP_MIN_BLOCKS_POLY_WARP 5
#endif
#ifndef RP3DG_NP_MIN_BLOCKS_POLY_THREAD
#define RP3DG_NP_MIN_BLOCKS_POLY_THREAD 4
#endif

namespace rp3dg {

// Internal kernel id: the per-thread half of the polyhedron schedule.
constexpr int ALGO_POLY_PER_THREAD = 7;
constexpr int NP_MIN_BLOCKS = RP3DG_NP_MIN_BLOCKS;
constexpr int NP_MIN_BLOCKS_POLY_WARP = RP3DG_NP_MIN_BLOCKS_POLY_WARP;
constexpr int NP_MIN_BLOCKS_POLY_THREAD = RP3DG_NP_MIN_BLOCKS_POLY_THREAD;

__constant__ BoxTables c_box_tables;

void upload_box_tables(const BoxTables& t, cudaStream_t s) {
    cudaMemcpyToSymbolAsync(c_box_tables, &t, sizeof(BoxTables), 0, cudaMemcpyHostToDevice, s);
}

struct ShapeRec {
    float4 params;
    int kind, mesh;
};

RD ShapeRec load_shape(const rp3dg_shape* shapes, int32_t idx) {
    const float4* p = reinterpret_cast<const float4*>(shapes + idx);
    const int4* k = reinterpret_cast<const int4*>(shapes + idx) + 1;
    ShapeRec s;
    s.params = __ldg(p);
    const int4 kk = __ldg(k);
    s.kind = kk.x;
    s.mesh = kk.y;
    return s;
}

// The shape kinds an algorithm batch accepts (CollisionDispatch::selectAlgorithm,
// CollisionDispatch.cpp:80-115); any other pair is reported as a bad shape.
RD bool is_poly_kind(int k) { return k == RP3DG_SHAPE_BOX || k == RP3DG_SHAPE_CONVEX_MESH; }
RD bool kinds_match(int algo, int k1, int k2) {
    switch (algo) {
        case RP3DG_ALGO_SPHERE_VS_SPHERE: return k1 == RP3DG_SHAPE_SPHERE && k2 == RP3DG_SHAPE_SPHERE;
        case RP3DG_ALGO_SPHERE_VS_CAPSULE:
            return (k1 == RP3DG_SHAPE_SPHERE && k2 == RP3DG_SHAPE_CAPSULE) || (k1 == RP3DG_SHAPE_CAPSULE && k2 == RP3DG_SHAPE_SPHERE);
        case RP3DG_ALGO_CAPSULE_VS_CAPSULE: return k1 == RP3DG_SHAPE_CAPSULE && k2 == RP3DG_SHAPE_CAPSULE;
        case RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON:
            return (k1 == RP3DG_SHAPE_SPHERE && is_poly_kind(k2)) || (is_poly_kind(k1) && k2 == RP3DG_SHAPE_SPHERE);
        case RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON:
            return (k1 == RP3DG_SHAPE_CAPSULE && is_poly_kind(k2)) || (is_poly_kind(k1) && k2 == RP3DG_SHAPE_CAPSULE);
        default: return is_poly_kind(k1) && is_poly_kind(k2);
    }
}

RD MeshPoly mesh_poly(const uint32_t* words, int32_t inst) {
    MeshPoly m;
    m.h = reinterpret_cast<const MeshHdr*>(words) + inst;
    m.w = words;
    return m;
}

RD BoxPoly box_poly(const ShapeRec& s, const BoxTables* t) {
    BoxPoly b;
    b.he = V(s.params.x, s.params.y, s.params.z);
    b.t = t;
    return b;
}

// Load one pair's inputs into an Item (every lane of a warp may call this for
// the same pair: the loads are broadcasts).
RD void load_item(const NpArgs& a, uint32_t i, Item& it) {
    const float4 p1 = a.pos1[i], q1 = a.rot1[i], p2 = a.pos2[i], q2 = a.rot2[i];
    it.t1 = X(V(p1.x, p1.y, p1.z), Q(q1.x, q1.y, q1.z, q1.w));
    it.t2 = X(V(p2.x, p2.y, p2.z), Q(q2.x, q2.y, q2.z, q2.w));
    it.report = a.report ? a.report[i] != 0 : true;
    it.colliding = false;
    it.gjk_capped = false;
    it.proposal = MLP_NO_PROPOSAL;
    it.proposal_tested = it.proposal_confirmed = false;
    if (a.cache) {
        const uint4 c = reinterpret_cast<const uint4*>(a.cache)[i];
        it.lf.gjk_axis = V(__uint_as_float(c.x), __uint_as_float(c.y), __uint_as_float(c.z));
        it.lf.flags = c.w & 0xffu;
        it.lf.sat_face = (c.w >> 8) & 0xffu;
        it.lf.sat_e1 = (c.w >> 16) & 0xffu;
        it.lf.sat_e2 = (c.w >> 24) & 0xffu;
    } else {
        it.lf.gjk_axis = V(0.0f, 1.0f, 0.0f);
        it.lf.flags = 0;
        it.lf.sat_face = it.lf.sat_e1 = it.lf.sat_e2 = 0;
    }
    it.out.nd = a.normal_depth;
    it.out.l1 = a.local1;
    it.out.l2 = a.local2;
    it.out.n = a.n;
    it.out.i = i;
    it.out.max = a.max_contacts;
    it.out.count = 0;
    it.out.first_normal = V(0.0f, 0.0f, 0.0f);
    it.out.first_depth = 0.0f;
    it.tri_side = 0;
    it.tri = nullptr;
    NP_EV_ONLY(for (uint32_t e = 0; e < NP_EVENT_COUNT; e++) it.ev[e] = 0u;)
}

RD void store_item(const NpArgs& a, uint32_t i, const Item& it) {
    if (it.gjk_capped) atomicOr(a.error, 2u);
#ifdef RP3DG_COUNT_EVENTS
    if (a.events)
        for (uint32_t e = 0; e < NP_EVENT_USED; e++)
            if (it.ev[e]) atomicAdd(a.events + e, (unsigned long long)it.ev[e]);
#endif
    a.is_colliding[i] = it.colliding ? 1 : 0;
    a.nb_contacts[i] = uint8_t(it.out.count < a.max_contacts ? it.out.count : a.max_contacts);
    if (a.cache) {
        uint4 c;
        c.x = __float_as_uint(it.lf.gjk_axis.x);
        c.y = __float_as_uint(it.lf.gjk_axis.y);
        c.z = __float_as_uint(it.lf.gjk_axis.z);
        c.w = (it.lf.flags & 0xffu) | ((it.lf.sat_face & 0xffu) << 8) | ((it.lf.sat_e1 & 0xffu) << 16) |
              ((it.lf.sat_e2 & 0xffu) << 24);
        reinterpret_cast<uint4*>(a.cache)[i] = c;
    }
}

// Returns bit 0 = a learned proposal was tested, bit 1 = it was confirmed.
template <int ALGO>
RD uint32_t process_pair(const NpArgs& a, uint32_t i, const BoxTables* box, const uint32_t* mesh_words,
                         uint32_t proposal = MLP_NO_PROPOSAL) {
    const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
    if (uint32_t(i1) >= a.nb_shapes || uint32_t(i2) >= a.nb_shapes) {
        // a pair naming a shape outside the table is reported as not colliding
        a.is_colliding[i] = 0;
        a.nb_contacts[i] = 0;
        atomicOr(a.error, 1u);
        return 0;
    }
    const ShapeRec s1 = load_shape(a.shapes, i1);
    const ShapeRec s2 = load_shape(a.shapes, i2);
    constexpr int CHECK = ALGO == ALGO_POLY_PER_THREAD ? int(RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON) : ALGO;
    if (!kinds_match(CHECK, s1.kind, s2.kind)) {
        // a pair the algorithm does not handle (a concave shape has no pair
        // test of its own: it goes through the middle phase's triangles)
        a.is_colliding[i] = 0;
        a.nb_contacts[i] = 0;
        atomicOr(a.error, 1u);
        return 0;
    }
    Item it;
    load_item(a, i, it);
    it.proposal = proposal;

    if (ALGO == RP3DG_ALGO_SPHERE_VS_SPHERE) {
        sphere_sphere(it, s1.params.x, s2.params.x);
    } else if (ALGO == RP3DG_ALGO_SPHERE_VS_CAPSULE) {
        const bool sphere1 = s1.kind == RP3DG_SHAPE_SPHERE;
        const ShapeRec& ss = sphere1 ? s1 : s2;
        const ShapeRec& cs = sphere1 ? s2 : s1;
        sphere_capsule(it, sphere1, SphereS{ss.params.x}, CapsuleS{cs.params.x, cs.params.y});
    } else if (ALGO == RP3DG_ALGO_CAPSULE_VS_CAPSULE) {
        capsule_capsule(it, CapsuleS{s1.params.x, s1.params.y}, CapsuleS{s2.params.x, s2.params.y});
    } else if (ALGO == RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON) {
        const bool sphere1 = s1.kind == RP3DG_SHAPE_SPHERE;
        const ShapeRec& ss = sphere1 ? s1 : s2;
        const ShapeRec& ps = sphere1 ? s2 : s1;
        if (ps.kind == RP3DG_SHAPE_BOX) sphere_poly(it, sphere1, SphereS{ss.params.x}, box_poly(ps, box));
        else sphere_poly(it, sphere1, SphereS{ss.params.x}, mesh_poly(mesh_words, ps.mesh));
    } else if (ALGO == RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON) {
        const bool cap1 = s1.kind == RP3DG_SHAPE_CAPSULE;
        const ShapeRec& cs = cap1 ? s1 : s2;
        const ShapeRec& ps = cap1 ? s2 : s1;
        const CapsuleS cap{cs.params.x, cs.params.y};
        if (ps.kind == RP3DG_SHAPE_BOX) capsule_poly(it, cap1, cap, box_poly(ps, box));
        else capsule_poly(it, cap1, cap, mesh_poly(mesh_words, ps.mesh));
    } else if (ALGO == ALGO_POLY_PER_THREAD) {
        // the thread-per-pair launch is given box-box pairs only
        sat_poly_poly(it, box_poly(s1, box), box_poly(s2, box), a.clip);
        it.lf.set(RP3DG_LF_WAS_USING_SAT, true);
        it.lf.set(RP3DG_LF_WAS_USING_GJK, false);
    } else {
        const bool b1 = s1.kind == RP3DG_SHAPE_BOX, b2 = s2.kind == RP3DG_SHAPE_BOX;
        if (b1 && b2) sat_poly_poly(it, box_poly(s1, box), box_poly(s2, box), a.clip);
        else if (!b1 && b2) sat_poly_poly(it, mesh_poly(mesh_words, s1.mesh), box_poly(s2, box), a.clip);
        else if (b1 && !b2) sat_poly_poly(it, box_poly(s1, box), mesh_poly(mesh_words, s2.mesh), a.clip);
        else sat_poly_poly(it, mesh_poly(mesh_words, s1.mesh), mesh_poly(mesh_words, s2.mesh), a.clip);
        // ConvexPolyhedronVsConvexPolyhedronAlgorithm.cpp:53-61
        it.lf.set(RP3DG_LF_WAS_USING_SAT, true);
        it.lf.set(RP3DG_LF_WAS_USING_GJK, false);
    }

    store_item(a, i, it);
    return (it.proposal_tested ? 1u : 0u) | (it.proposal_confirmed ? 2u : 0u);
}

// One triangle test of a convex vs concave pair (the narrow-phase input that
// computeConvexVsConcaveMiddlePhase creates per overlapping triangle,
// CollisionDetectionSystem.cpp:522-615): the convex shape comes from the
// shape table, the TriangleShape from args.tri.
template <int ALGO>
RD void process_tri(const NpArgs& a, uint32_t i, const BoxTables* box, const uint32_t* mesh_words) {
    const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
    const bool tri1 = i1 < 0;
    const int32_t ci = tri1 ? i2 : i1;
    bool ok = (i1 < 0) != (i2 < 0) && uint32_t(ci) < a.nb_shapes;
    ShapeRec cs;
    if (ok) {
        cs = load_shape(a.shapes, ci);
        ok = ALGO == RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON    ? cs.kind == RP3DG_SHAPE_SPHERE
             : ALGO == RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON ? cs.kind == RP3DG_SHAPE_CAPSULE
                                                               : is_poly_kind(cs.kind);
    }
    if (!ok) {
        a.is_colliding[i] = 0;
        a.nb_contacts[i] = 0;
        atomicOr(a.error, 1u);
        return;
    }
    TriPoly tp;
    const float4 f0 = a.tri[i], f1 = a.tri[size_t(a.n) + i], f2 = a.tri[2 * size_t(a.n) + i];
    const float4 f3 = a.tri[3 * size_t(a.n) + i], f4 = a.tri[4 * size_t(a.n) + i];
    const float4 f5 = a.tri[5 * size_t(a.n) + i], f6 = a.tri[6 * size_t(a.n) + i];
    tp.p0 = V(f0.x, f0.y, f0.z);
    tp.p1 = V(f1.x, f1.y, f1.z);
    tp.p2 = V(f2.x, f2.y, f2.z);
    tp.n = V(f3.x, f3.y, f3.z);
    tp.vn0 = V(f4.x, f4.y, f4.z);
    tp.vn1 = V(f5.x, f5.y, f5.z);
    tp.vn2 = V(f6.x, f6.y, f6.z);
    tp.t = box;
    Item it;
    load_item(a, i, it);
    it.tri_side = tri1 ? 1u : 2u;
    it.tri = &tp;
    if (ALGO == RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON) {
        sphere_poly(it, !tri1, SphereS{cs.params.x}, tp);
    } else if (ALGO == RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON) {
        capsule_poly(it, !tri1, CapsuleS{cs.params.x, cs.params.y}, tp);
    } else {
        if (cs.kind == RP3DG_SHAPE_BOX) {
            if (tri1) sat_poly_poly(it, tp, box_poly(cs, box), a.clip);
            else sat_poly_poly(it, box_poly(cs, box), tp, a.clip);
        } else {
            if (tri1) sat_poly_poly(it, tp, mesh_poly(mesh_words, cs.mesh), a.clip);
            else sat_poly_poly(it, mesh_poly(mesh_words, cs.mesh), tp, a.clip);
        }
        // ConvexPolyhedronVsConvexPolyhedronAlgorithm.cpp:53-61
        it.lf.set(RP3DG_LF_WAS_USING_SAT, true);
        it.lf.set(RP3DG_LF_WAS_USING_GJK, false);
    }
    store_item(a, i, it);
}

// Shape combinations of the polyhedron pairs a warp-per-pair launch takes:
// each launch is compiled for one, so it carries one SAT instantiation
// (fewer registers, a smaller code footprint)
constexpr int COMBO_MESH_BOX = 1, COMBO_BOX_MESH = 2, COMBO_MESH_MESH = 3;

// Convex polyhedron vs convex polyhedron, one warp per pair, for pairs of
// shape combination COMBO.
template <int COMBO>
RD uint32_t process_pair_warp(const NpArgs& a, uint32_t i, int lane, const BoxTables* box, const uint32_t* mesh_words,
                              WarpScratch& stage, uint32_t proposal) {
    const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
    if (uint32_t(i1) >= a.nb_shapes || uint32_t(i2) >= a.nb_shapes) {
        if (lane == 0) {
            a.is_colliding[i] = 0;
            a.nb_contacts[i] = 0;
            atomicOr(a.error, 1u);
        }
        return 0;
    }
    const ShapeRec s1 = load_shape(a.shapes, i1);
    const ShapeRec s2 = load_shape(a.shapes, i2);
    if (!kinds_match(RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON, s1.kind, s2.kind)) {
        if (lane == 0) {
            a.is_colliding[i] = 0;
            a.nb_contacts[i] = 0;
            atomicOr(a.error, 1u);
        }
        return 0;
    }
    Item it;
    load_item(a, i, it);
    it.proposal = proposal;
    if constexpr (COMBO == COMBO_MESH_BOX)
        warp_sat_poly_poly(it, mesh_poly(mesh_words, s1.mesh), box_poly(s2, box), a.clip, lane, stage);
    else if constexpr (COMBO == COMBO_BOX_MESH)
        warp_sat_poly_poly(it, box_poly(s1, box), mesh_poly(mesh_words, s2.mesh), a.clip, lane, stage);
    else
        warp_sat_poly_poly(it, mesh_poly(mesh_words, s1.mesh), mesh_poly(mesh_words, s2.mesh), a.clip, lane, stage);
    // ConvexPolyhedronVsConvexPolyhedronAlgorithm.cpp:53-61
    it.lf.set(RP3DG_LF_WAS_USING_SAT, true);
    it.lf.set(RP3DG_LF_WAS_USING_GJK, false);
    if (lane == 0) store_item(a, i, it);
    return (it.proposal_tested ? 1u : 0u) | (it.proposal_confirmed ? 2u : 0u);
}

// MLP input features of a polyhedron pair (zero for a pair that is not one).
RD void pair_features(const NpArgs& a, uint32_t i, const BoxTables* box, const uint32_t* mesh_words, float* f) {
    for (int k = 0; k < 32; k++) f[k] = 0.0f;
    if (i >= a.n) return;
    const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
    if (uint32_t(i1) >= a.nb_shapes || uint32_t(i2) >= a.nb_shapes) return;
    const ShapeRec s1 = load_shape(a.shapes, i1), s2 = load_shape(a.shapes, i2);
    if (!is_poly_kind(s1.kind) || !is_poly_kind(s2.kind)) return;
    const float4 p1 = a.pos1[i], q1 = a.rot1[i], p2 = a.pos2[i], q2 = a.rot2[i];
    const xform t1 = X(V(p1.x, p1.y, p1.z), Q(q1.x, q1.y, q1.z, q1.w));
    const xform t2 = X(V(p2.x, p2.y, p2.z), Q(q2.x, q2.y, q2.z, q2.w));
    const bool b1 = s1.kind == RP3DG_SHAPE_BOX, b2 = s2.kind == RP3DG_SHAPE_BOX;
    float g[MLP_IN];
    if (b1 && b2) axis_features(t1, t2, box_poly(s1, box), box_poly(s2, box), false, g);
    else if (!b1 && b2) axis_features(t1, t2, mesh_poly(mesh_words, s1.mesh), box_poly(s2, box), true, g);
    else if (b1 && !b2) axis_features(t1, t2, box_poly(s1, box), mesh_poly(mesh_words, s2.mesh), false, g);
    else axis_features(t1, t2, mesh_poly(mesh_words, s1.mesh), mesh_poly(mesh_words, s2.mesh), true, g);
    for (int k = 0; k < MLP_IN; k++) f[k] = g[k];
}

template <int ALGO>
struct MinBlocks { static constexpr int value = NP_MIN_BLOCKS; };
template <>
struct MinBlocks<RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON> { static constexpr int value = NP_MIN_BLOCKS_POLY_WARP; };
template <>
struct MinBlocks<ALGO_POLY_PER_THREAD> { static constexpr int value = NP_MIN_BLOCKS_POLY_THREAD; };

template <int ALGO>
__global__ void __launch_bounds__(NP_BLOCK, MinBlocks<ALGO>::value) narrowphase_kernel(const NpArgs a) {
    extern __shared__ uint32_t s_mesh[];
    __shared__ BoxTables s_box;
    constexpr bool uses_poly = ALGO >= RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON;
    const uint32_t* mesh_words = a.mesh_words;
    if (uses_poly) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&c_box_tables);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&s_box);
        for (uint32_t k = threadIdx.x; k < sizeof(BoxTables) / 4; k += blockDim.x) dst[k] = src[k];
        if (a.stage_mesh && ALGO != ALGO_POLY_PER_THREAD) {
            for (uint32_t k = threadIdx.x; k < a.mesh_nwords; k += blockDim.x) s_mesh[k] = __ldg(a.mesh_words + k);
            mesh_words = s_mesh;
        }
        __syncthreads();
    }
    if constexpr (ALGO == ALGO_POLY_PER_THREAD) {
        // Polyhedron pairs by tiles of 32 (in the class order of the pair
        // order perm): the box-box pairs of a tile (12 x 12 edge pairs) are
        // done one per thread here; a pair with a convex mesh (up to 128 x 128
        // edge pairs) is appended to the list of its shape combination, which
        // a warp-per-pair launch of that combination then takes.
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const uint32_t nwarps = gridDim.x * (NP_BLOCK / 32);
        uint32_t tested = 0, confirmed = 0;
        for (uint32_t tile = blockIdx.x * (NP_BLOCK / 32) + warp; tile * 32u < a.n; tile += nwarps) {
            const uint32_t t = tile * 32u + lane;
            const uint32_t i = (a.perm && t < a.n) ? a.perm[t] : t;
            int combo = 0;   // box-box, or a pair whose check fails in process_pair
            if (t < a.n) {
                const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
                if (uint32_t(i1) < a.nb_shapes && uint32_t(i2) < a.nb_shapes) {
                    const ShapeRec r1 = load_shape(a.shapes, i1), r2 = load_shape(a.shapes, i2);
                    if (is_poly_kind(r1.kind) && is_poly_kind(r2.kind)) {
                        const bool b1 = r1.kind == RP3DG_SHAPE_BOX, b2 = r2.kind == RP3DG_SHAPE_BOX;
                        combo = (b1 && b2) ? 0 : (!b1 && b2) ? COMBO_MESH_BOX : (b1 ? COMBO_BOX_MESH : COMBO_MESH_MESH);
                    }
                }
            }
            for (int c = COMBO_MESH_BOX; c <= COMBO_MESH_MESH; c++) {
                const uint32_t m = __ballot_sync(FULL_MASK, combo == c);
                if (!m) continue;
                const int leader = __ffs(m) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(a.work + (c - 1), uint32_t(__popc(m)));
                base = __shfl_sync(FULL_MASK, base, leader);
                if (combo == c) a.plist[size_t(c - 1) * a.n + base + uint32_t(__popc(m & ((1u << lane) - 1u)))] = i;
            }
            uint32_t proposal = MLP_NO_PROPOSAL;
            if (a.proposals && t < a.n) {
                proposal = a.proposals[i];
                if (proposal >= MLP_OUT) proposal = MLP_NO_PROPOSAL;
            }
            uint32_t r = 0;
            if (t < a.n && combo == 0)
                r = process_pair<ALGO_POLY_PER_THREAD>(a, i, &s_box, mesh_words, proposal);
            tested += __popc(__ballot_sync(FULL_MASK, r & 1u));
            confirmed += __popc(__ballot_sync(FULL_MASK, (r & 2u) != 0));
        }
        if (a.mlp_stats && lane == 0 && tested) {
            atomicAdd(&a.mlp_stats[0], (unsigned long long)tested);
            atomicAdd(&a.mlp_stats[1], (unsigned long long)confirmed);
        }
    } else {
        const uint32_t stride = gridDim.x * blockDim.x;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride)
            process_pair<ALGO>(a, i, &s_box, mesh_words);
    }
}

// The pairs with a convex mesh of one shape combination, listed by the
// thread-per-pair launch: persistent warps take them one at a time (so the
// launch ends within one pair's time of its average), faces over lanes
// (ballot / arg-min), edge staging in shared memory, the Gauss-map pass and
// the edge distances 32 at a time, warp-parallel clipping.
template <int COMBO>
__global__ void __launch_bounds__(NP_BLOCK, NP_MIN_BLOCKS_POLY_WARP) narrowphase_warp_kernel(const NpArgs a) {
    extern __shared__ uint32_t s_mesh[];
    __shared__ BoxTables s_box;
    __shared__ WarpScratch s_stage[NP_BLOCK / 32];
    const uint32_t total = __ldcg(a.work + (COMBO - 1));
    if (total == 0) return;   // uniform: nothing of this combination in the batch
    const uint32_t* mesh_words = a.mesh_words;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&c_box_tables);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&s_box);
        for (uint32_t k = threadIdx.x; k < sizeof(BoxTables) / 4; k += blockDim.x) dst[k] = src[k];
        if (a.stage_mesh) {
            for (uint32_t k = threadIdx.x; k < a.mesh_nwords; k += blockDim.x) s_mesh[k] = __ldg(a.mesh_words + k);
            mesh_words = s_mesh;
        }
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpScratch& ws = s_stage[warp];
    const uint32_t* list = a.plist + size_t(COMBO - 1) * a.n;
    uint32_t tested = 0, confirmed = 0;
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(a.work + 3 + (COMBO - 1), 1u);
        k = __shfl_sync(FULL_MASK, k, 0);
        if (k >= total) break;
        const uint32_t i = list[k];
        uint32_t proposal = a.proposals ? uint32_t(a.proposals[i]) : uint32_t(MLP_NO_PROPOSAL);
        if (proposal >= MLP_OUT) proposal = MLP_NO_PROPOSAL;
        const uint32_t r = process_pair_warp<COMBO>(a, i, lane, &s_box, mesh_words, ws, proposal);
        tested += r & 1u;
        confirmed += (r >> 1) & 1u;
        __syncwarp();
    }
    if (a.mlp_stats && lane == 0 && tested) {
        atomicAdd(&a.mlp_stats[0], (unsigned long long)tested);
        atomicAdd(&a.mlp_stats[1], (unsigned long long)confirmed);
    }
}

template <int ALGO>
__global__ void __launch_bounds__(NP_BLOCK, NP_MIN_BLOCKS) narrowphase_tri_kernel(const NpArgs a) {
    extern __shared__ uint32_t s_mesh[];
    __shared__ BoxTables s_box;
    const uint32_t* mesh_words = a.mesh_words;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&c_box_tables);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&s_box);
        for (uint32_t k = threadIdx.x; k < sizeof(BoxTables) / 4; k += blockDim.x) dst[k] = src[k];
        if (a.stage_mesh) {
            for (uint32_t k = threadIdx.x; k < a.mesh_nwords; k += blockDim.x) s_mesh[k] = __ldg(a.mesh_words + k);
            mesh_words = s_mesh;
        }
        __syncthreads();
    }
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride)
        process_tri<ALGO>(a, i, &s_box, mesh_words);
}

cudaError_t launch_narrowphase_tri(int algo, const NpArgs& args, int num_sms, cudaStream_t stream) {
    if (args.n == 0) return cudaSuccess;
    const void* k = algo == RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON
                        ? reinterpret_cast<const void*>(&narrowphase_tri_kernel<RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON>)
                    : algo == RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON
                        ? reinterpret_cast<const void*>(&narrowphase_tri_kernel<RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON>)
                    : algo == RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON
                        ? reinterpret_cast<const void*>(&narrowphase_tri_kernel<RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON>)
                        : nullptr;
    if (!k || !args.tri) return cudaErrorInvalidValue;
    const size_t smem = args.stage_mesh ? size_t(args.mesh_nwords) * 4 : 0;
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k);
    if (e != cudaSuccess) return e;
    if (smem > 0 && fa.sharedSizeBytes + smem > 48 * 1024) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    const uint32_t blocks_needed = (args.n + NP_BLOCK - 1) / NP_BLOCK;
    const uint32_t cap = uint32_t(num_sms) * 16u;
    const uint32_t blocks = blocks_needed < cap ? blocks_needed : cap;
    void* params[] = {const_cast<NpArgs*>(&args)};
    return cudaLaunchKernel(k, dim3(blocks), dim3(NP_BLOCK), params, smem, stream);
}

// Counting sort of a polyhedron batch's pairs by learned class, so that a
// tile of 32 pairs holds pairs of one class: the predicted-colliding pairs
// (class 15: full SAT and clipping) share tiles, and pairs whose proposal
// the exact test confirms share tiles and finish together.  Only the order in
// which the pairs are processed changes (each pair writes its own slots), so
// the results do not depend on it; the order inside a class follows the
// atomics.  Rank of class c: 15 first, then 0..14.
__device__ __forceinline__ uint32_t class_rank(uint32_t c) { return c >= 15u ? 0u : c + 1u; }
__global__ void __launch_bounds__(256) partition_count(const NpArgs a, const uint8_t* __restrict__ cls,
                                                       uint32_t* __restrict__ counts) {
    const uint32_t n = a.n;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = i < n ? class_rank(cls[i]) : 16u;
    // a batch with a convex mesh keeps its order: its pairs go one per warp,
    // where grouping gains nothing
    if (i < n) {
        const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
        const bool box = uint32_t(i1) < a.nb_shapes && uint32_t(i2) < a.nb_shapes &&
                         load_shape(a.shapes, i1).kind == RP3DG_SHAPE_BOX && load_shape(a.shapes, i2).kind == RP3DG_SHAPE_BOX;
        if (!box) counts[31] = 1u;
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, r);
    const uint32_t lane = threadIdx.x & 31u;
    if (r < 16u && (peers & ((1u << lane) - 1u)) == 0) atomicAdd(counts + r, uint32_t(__popc(peers)));
}
__global__ void __launch_bounds__(256) partition_scatter(const uint8_t* __restrict__ cls, uint32_t n,
                                                         uint32_t* __restrict__ counts, uint32_t* __restrict__ perm) {
    __shared__ uint32_t base[16];
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int k = 0; k < 16; k++) { base[k] = run; run += counts[k]; }
    }
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (counts[31]) {
        if (i < n) perm[i] = i;
        return;
    }
    const uint32_t r = i < n ? class_rank(cls[i]) : 16u;
    const uint32_t peers = __match_any_sync(0xffffffffu, r);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t rank = uint32_t(__popc(peers & ((1u << lane) - 1u)));
    const uint32_t leader = uint32_t(__ffs(peers)) - 1u;
    uint32_t off = 0;
    if (r < 16u && lane == leader) off = atomicAdd(counts + 16 + r, uint32_t(__popc(peers)));
    off = __shfl_sync(0xffffffffu, off, int(leader));
    if (r < 16u) perm[base[r] + off + rank] = i;
}
cudaError_t launch_partition_by_class(const NpArgs& a, const uint8_t* cls, uint32_t* counts, uint32_t* perm,
                                      cudaStream_t stream) {
    const uint32_t n = a.n;
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(counts, 0, 32 * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    const uint32_t nb = (n + 255) / 256;
    partition_count<<<nb, 256, 0, stream>>>(a, cls, counts);
    partition_scatter<<<nb, 256, 0, stream>>>(cls, n, counts, perm);
    return cudaGetLastError();
}

// Classification of a polyhedron batch before its SAT kernels, per tile of
// 32 pairs (one warp):
//   - the geometric class of a box-box pair: its inscribed spheres overlap
//     (certainly colliding: full SAT and clipping), its bounding spheres are
//     apart (certainly separated: a face test ends it), or neither, in which
//     case a valid last-frame record predicts it (was colliding / separated
//     by a SAT axis); a pair with a mesh gets its own class, so that box
//     tiles stay all-box for the thread-per-pair kernel;
//   - with the learned proposal on, the warp also computes the pairs'
//     features and runs the MLP on the bf16 tensor cores (mma.sync
//     m16n8k16, 112 MMAs per tile) and writes each pair's proposed feature
//     (15 = none) to `proposals`, which the SAT kernels test exactly.
// `key` receives the order class that partition_count / partition_scatter
// sort by (class 15 first, then 0..14): certainly colliding (15), uncertain
// (0), certainly separated (1) and mesh pairs (2); the learned proposals do
// not change the order.  Only the order in which the pairs are processed
// depends on the key.
RD uint8_t box_pair_class(const NpArgs& a, uint32_t i) {
    if (i >= a.n) return 0;
    const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
    if (uint32_t(i1) >= a.nb_shapes || uint32_t(i2) >= a.nb_shapes) return 0;
    const ShapeRec r1 = load_shape(a.shapes, i1), r2 = load_shape(a.shapes, i2);
    if (r1.kind != RP3DG_SHAPE_BOX || r2.kind != RP3DG_SHAPE_BOX) return 2;   // a mesh pair: its own tiles
    const float4 p1 = a.pos1[i], p2 = a.pos2[i];
    const float dx = p2.x - p1.x, dy = p2.y - p1.y, dz = p2.z - p1.z;
    const float d2 = dx * dx + dy * dy + dz * dz;
    const float4 h1 = r1.params, h2 = r2.params;
    const float R = sqrtf(h1.x * h1.x + h1.y * h1.y + h1.z * h1.z) + sqrtf(h2.x * h2.x + h2.y * h2.y + h2.z * h2.z);
    const float r = fminf(h1.x, fminf(h1.y, h1.z)) + fminf(h2.x, fminf(h2.y, h2.z));
    return d2 > R * R * 1.0001f ? 1 : (d2 < r * r * 0.9999f ? 15 : 0);
}

__global__ void __launch_bounds__(NP_BLOCK) classify_pairs(const NpArgs a, uint8_t* __restrict__ key,
                                                           uint8_t* __restrict__ proposals) {
    __shared__ float s_feat[NP_BLOCK / 32][32][MLP_KPAD];
    __shared__ uint32_t s_cls[NP_BLOCK / 32][32];
    __shared__ BoxTables s_box;
    const bool learned = a.mlp != nullptr && proposals != nullptr;
    if (learned) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&c_box_tables);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&s_box);
        for (uint32_t k = threadIdx.x; k < sizeof(BoxTables) / 4; k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nwarps = gridDim.x * (NP_BLOCK / 32);
    for (uint32_t tile = blockIdx.x * (NP_BLOCK / 32) + warp; tile * 32u < a.n; tile += nwarps) {
        const uint32_t i = tile * 32u + lane;
        uint8_t geo = box_pair_class(a, i);
        // an uncertain box pair with a last-frame record follows last
        // frame's outcome: colliding pairs clip, SAT-separated ones usually
        // end at the remembered axis
        if (geo == 0 && i < a.n && a.cache) {
            const uint8_t f = a.cache[i].flags;
            if (f & RP3DG_LF_IS_VALID) geo = (f & RP3DG_LF_WAS_COLLIDING) ? 15 : ((f & RP3DG_LF_WAS_USING_SAT) ? 1 : 0);
        }
        uint8_t k = geo;
        if (learned) {
            // a proposal is only looked at where the full SAT starts: not for
            // pairs that certainly collide or are certainly apart (geometric
            // class), nor, mostly, for pairs whose SAT cache from the last
            // frame is tested first; a tile none of whose pairs needs one
            // skips the features and the MLP
            bool need = i < a.n && (geo == 0 || geo == 2);
            if (need && a.cache) {
                const uint8_t f = a.cache[i].flags;
                if ((f & RP3DG_LF_IS_VALID) && (f & RP3DG_LF_WAS_USING_SAT)) need = false;
            }
            uint32_t c = MLP_NO_PROPOSAL;
            if (__any_sync(0xffffffffu, need)) {
                pair_features(a, i, &s_box, a.mesh_words, s_feat[warp][lane]);
                __syncwarp();
                c = mlp_infer_tile(s_feat[warp], *static_cast<const MlpPacked*>(a.mlp), lane, s_cls[warp]);
                if (c >= MLP_OUT || !need) c = MLP_NO_PROPOSAL;
                __syncwarp();
            }
            if (i < a.n) proposals[i] = uint8_t(c);
        }
        if (i < a.n) key[i] = k;
    }
}

// One warp per 32 pairs: an inclusive scan of the counts, one atomic for
// the group's first record, then the warp writes its records as one
// contiguous run (lane l the float4s l, l + 32, ...), so that records in
// page-locked host memory go over the bus in full-width writes.  Float4 j
// of the run belongs to record r = j / 3 of the lane whose inclusive count
// is the first above r.
__global__ void __launch_bounds__(256) compact_contacts(const CompactArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u, group = i >> 5;
    if ((group << 5) >= a.n) return;   // whole warps leave together
    const uint32_t c = i < a.n ? a.nb[i] : 0u;
    uint32_t incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= uint32_t(d)) incl += v;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t start = 0;
    if (lane == 0) {
        start = total ? atomicAdd(a.counter, total) : 0u;
        a.warp_start[group] = start;
    }
    start = __shfl_sync(0xffffffffu, start, 0);
    float4* dst = a.records + 3 * size_t(start);
    const uint32_t excl = incl - c;
    for (uint32_t j0 = 0; j0 < 3 * total; j0 += 32) {
        const uint32_t j = j0 + lane, r = j / 3u, part = j - 3u * r;
        uint32_t p = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1)
            if (__shfl_sync(0xffffffffu, incl, int(p + step - 1)) <= r) p += step;
        const uint32_t k = r - __shfl_sync(0xffffffffu, excl, int(p));
        if (j < 3 * total) {
            const size_t o = size_t(k) * a.n + (size_t(group) << 5) + p;
            dst[j] = part == 0 ? a.nd[o] : (part == 1 ? a.l1[o] : a.l2[o]);
        }
    }
}

cudaError_t launch_compact_contacts(const CompactArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    compact_contacts<<<(a.n + 255) / 256, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_classify_pairs(const NpArgs& args, uint8_t* key, uint8_t* proposals, int num_sms,
                                  cudaStream_t stream) {
    if (args.n == 0) return cudaSuccess;
    const uint32_t blocks_needed = (args.n + NP_BLOCK - 1) / NP_BLOCK;
    const uint32_t cap = uint32_t(num_sms) * 16u;
    classify_pairs<<<blocks_needed < cap ? blocks_needed : cap, NP_BLOCK, 0, stream>>>(args, key, proposals);
    return cudaGetLastError();
}

static const void* kernel_ptr(int algo) {
    switch (algo) {
        case 1: return reinterpret_cast<const void*>(&narrowphase_kernel<1>);
        case 2: return reinterpret_cast<const void*>(&narrowphase_kernel<2>);
        case 3: return reinterpret_cast<const void*>(&narrowphase_kernel<3>);
        case 4: return reinterpret_cast<const void*>(&narrowphase_kernel<4>);
        case 5: return reinterpret_cast<const void*>(&narrowphase_kernel<5>);
        case 8 + COMBO_MESH_BOX: return reinterpret_cast<const void*>(&narrowphase_warp_kernel<COMBO_MESH_BOX>);
        case 8 + COMBO_BOX_MESH: return reinterpret_cast<const void*>(&narrowphase_warp_kernel<COMBO_BOX_MESH>);
        case 8 + COMBO_MESH_MESH: return reinterpret_cast<const void*>(&narrowphase_warp_kernel<COMBO_MESH_MESH>);
        case ALGO_POLY_PER_THREAD: return reinterpret_cast<const void*>(&narrowphase_kernel<ALGO_POLY_PER_THREAD>);
    }
    return nullptr;
}

#ifdef RP3DG_PROFILE_PHASES
// Profiling builds only: per-phase cycles (summed over warps) and counts of the
// warp-cooperative SAT; phases 0 = setup + temporal coherence, 1 = faces of
// polyhedron 1, 2 = faces of polyhedron 2, 3 = edge staging, 4 = edge pairs,
// 5 = contact generation.  clear != 0 zeroes the counters after reading.
extern "C" int rp3dg_profile_phases(unsigned long long* cycles, unsigned long long* counts, int clear) {
    cudaMemcpyFromSymbol(cycles, g_phase_cycles, sizeof(unsigned long long) * 8);
    cudaMemcpyFromSymbol(counts, g_phase_count, sizeof(unsigned long long) * 8);
    if (clear) {
        const unsigned long long z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z));
        cudaMemcpyToSymbol(g_phase_count, z, sizeof(z));
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}
#endif

static cudaError_t launch_one(int algo, const NpArgs& args, int num_sms, cudaStream_t stream);

cudaError_t launch_narrowphase(int algo, const NpArgs& args, int num_sms, cudaStream_t stream, int* launches) {
    *launches = 0;
    if (args.n == 0) return cudaSuccess;
    if (algo == RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON) {
        // the thread-per-pair launch (box-box pairs, and the lists of the
        // mesh pairs), then one warp-per-pair launch per shape combination
        if (!args.plist || !args.work) return cudaErrorInvalidValue;
        cudaError_t e = cudaMemsetAsync(args.work, 0, 6 * sizeof(uint32_t), stream);
        if (e != cudaSuccess) return e;
        e = launch_one(ALGO_POLY_PER_THREAD, args, num_sms, stream);
        if (e != cudaSuccess) return e;
        ++*launches;
        for (int c = COMBO_MESH_BOX; c <= COMBO_MESH_MESH; c++) {
            e = launch_one(8 + c, args, num_sms, stream);
            if (e != cudaSuccess) return e;
            ++*launches;
        }
        return cudaSuccess;
    }
    cudaError_t e = launch_one(algo, args, num_sms, stream);
    if (e == cudaSuccess) ++*launches;
    return e;
}

// Per kernel: its static shared memory, the dynamic size its opt-in was set
// for, and its resident CTAs per SM for that size (queried once: the
// queries cost more host time than a launch).
struct LaunchCache {
    bool known = false;
    size_t static_smem = 0, smem = ~size_t(0);
    int per_sm = 0;
};

static cudaError_t launch_one(int algo, const NpArgs& args, int num_sms, cudaStream_t stream) {
    const void* k = kernel_ptr(algo);
    if (!k) return cudaErrorInvalidValue;
    const bool warp_list = algo > 8;   // narrowphase_warp_kernel<algo - 8>
    size_t smem = (args.stage_mesh && algo != ALGO_POLY_PER_THREAD) ? size_t(args.mesh_nwords) * 4 : 0;
    static thread_local LaunchCache cache[16];
    LaunchCache& lc = cache[algo & 15];
    cudaError_t e = cudaSuccess;
    if (!lc.known) {
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, k);
        if (e != cudaSuccess) return e;
        lc.static_smem = fa.sharedSizeBytes;
        lc.known = true;
    }
    if (lc.smem != smem) {
        // static + dynamic shared memory above 48 KB needs the opt-in attribute
        if (smem > 0 && lc.static_smem + smem > 48 * 1024) {
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            if (e != cudaSuccess) return e;
        }
        lc.per_sm = 0;
        if (warp_list) {
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lc.per_sm, k, NP_BLOCK, smem);
            if (e != cudaSuccess) return e;
        }
        lc.smem = smem;
    }
    // a warp-per-pair launch can use a warp per pair (4 per CTA), the others a thread
    const uint32_t blocks_needed = warp_list ? (args.n + 3) / 4 : (args.n + NP_BLOCK - 1) / NP_BLOCK;
    // Enough CTAs to fill every SM several times; the grid-stride loop covers the rest.
    const uint32_t cap = uint32_t(num_sms) * 16u;
    uint32_t blocks = blocks_needed < cap ? blocks_needed : cap;
    if (warp_list) {
        // persistent: the CTAs that fit on the device at once
        const uint32_t resident = uint32_t(num_sms) * uint32_t(lc.per_sm > 0 ? lc.per_sm : 1);
        blocks = blocks_needed < resident ? blocks_needed : resident;
    }
    void* params[] = {const_cast<NpArgs*>(&args)};
    return cudaLaunchKernel(k, dim3(blocks), dim3(NP_BLOCK), params, smem, stream);
}

}  // namespace rp3dg

#ifdef RP3DG_COUNT_EVENTS
// Entry points of the event-counting build (this file compiled a second time
// by narrowphase_events.cu, which renames the namespace); args points to an
// NpArgs of the same layout with `events` set.
cudaError_t rp3dg_events_launch_narrowphase(int algo, const void* args, int num_sms, cudaStream_t stream, int* launches) {
    return rp3dg::launch_narrowphase(algo, *static_cast<const rp3dg::NpArgs*>(args), num_sms, stream, launches);
}
cudaError_t rp3dg_events_launch_narrowphase_tri(int algo, const void* args, int num_sms, cudaStream_t stream) {
    return rp3dg::launch_narrowphase_tri(algo, *static_cast<const rp3dg::NpArgs*>(args), num_sms, stream);
}
void rp3dg_events_upload_box_tables(const void* t, cudaStream_t stream) {
    rp3dg::upload_box_tables(*static_cast<const rp3dg::BoxTables*>(t), stream);
}
#endif
