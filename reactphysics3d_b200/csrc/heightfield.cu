// Convex vs concave middle phase for height fields, and the potential
// contact manifolds of those pairs (paths below are inside the reference
// project):
//   hf_rects:     the convex collider's AABB in the height field's space and
//                 the rectangle of grid cells it covers
//                 (CollisionDetectionSystem::computeConvexVsConcaveMiddlePhase,
//                 src/systems/CollisionDetectionSystem.cpp:522-615;
//                 HeightFieldShape::computeOverlappingTriangles,
//                 src/collision/shapes/HeightFieldShape.cpp:53-63;
//                 HeightField::computeMinMaxGridCoordinates,
//                 src/collision/HeightField.cpp:220-253)
//   concave meshes: the convex AABB without the mesh's scale queried
//                 against the mesh's triangle tree (ConcaveMeshShape::
//                 computeOverlappingTriangles, src/collision/shapes/
//                 ConcaveMeshShape.cpp:135-175): counted by hf_rects, listed
//                 in query order by hf_list
//   hf_tests:     one narrow-phase test per triangle of the rectangle, two
//                 per cell in (i, j) order (HeightField::computeOverlappingTriangles,
//                 HeightField.cpp:139-216; TriangleShape constructor,
//                 src/collision/shapes/TriangleShape.cpp:40-60), with its
//                 temporal-coherence record carried over from the previous
//                 step when the triangle was tested then
//                 (ConcaveOverlappingPair::addLastFrameInfoIfNecessary and
//                 clearObsoleteLastFrameInfos, OverlappingPairs.h:231-290)
//   hf_manifolds: the pair's contact points merged into potential manifolds
//                 by normal direction (processPotentialContacts, concave
//                 branch, CollisionDetectionSystem.cpp:1281-1375), the
//                 shallowest manifolds dropped down to four
//                 (reducePotentialContactManifolds, :1394-1430) and each
//                 manifold reduced to four points and de-duplicated
//                 (:1433-1458).
#include <cuda_runtime.h>

#include "hf_launch.h"
#include "manifold_reduce.cuh"
#include "rp3dg_math.cuh"
#include "shape_aabb.cuh"

namespace rp3dg {

namespace {

constexpr uint32_t MAXC = RP3DG_MAX_CONTACTS_PER_PAIR;
constexpr uint32_t MAX_POTENTIAL_MANIFOLDS = 64;     // NB_MAX_POTENTIAL_CONTACT_MANIFOLDS (configuration.h:140)
constexpr uint32_t MAX_POTENTIAL_POINTS = 255;       // NB_MAX_CONTACT_POINTS_IN_POTENTIAL_MANIFOLD (:143)

RD float fmax_std(float a, float b) { return (a < b) ? b : a; }  // std::max
RD float fmin_std(float a, float b) { return (b < a) ? b : a; }  // std::min
RD int clamp_int(int v, int lo, int hi) {                        // clamp (mathematics_functions.h:48-51)
    const int m = v < lo ? lo : v;
    return hi < m ? hi : m;
}

// The convex collider's AABB in the concave shape's local space
// (computeConvexVsConcaveMiddlePhase: convexShape->computeTransformedAABB of
// convexToConcaveTransform = concave^-1 * convex).
RD void convex_aabb_in_concave(const int4 it, const int32_t* c_shape, const rp3dg_shape* shapes,
                               const float4* bounds, const float4* c_wpos, const float4* c_wori, v3& amin,
                               v3& amax) {
    const float4 pv = c_wpos[it.x], qv = c_wori[it.x], pc = c_wpos[it.y], qc = c_wori[it.y];
    const xform tConvex = X(V(pv.x, pv.y, pv.z), Q(qv.x, qv.y, qv.z, qv.w));
    const xform tConcave = X(V(pc.x, pc.y, pc.z), Q(qc.x, qc.y, qc.z, qc.w));
    const xform c2c = xmul(xinv(tConcave), tConvex);
    const int32_t si = c_shape[it.x];
    const rp3dg_shape s = shapes[si];
    shape_transformed_aabb(s.kind, s.params[0], bounds[2 * si], bounds[2 * si + 1], c2c, amin, amax);
}

// ConcaveMeshShape::computeOverlappingTriangles (ConcaveMeshShape.cpp:135-175)
// over DynamicAABBTree::reportAllShapesOverlappingWithAABB (DynamicAABBTree.cpp:
// 641-681): the AABB without the mesh's scale (AABB::applyScale by
// decimal(1.0) / scale), then the leaves whose AABB it touches (inclusive
// test), children[1] popped before children[0].  `emit(k, triangle)` sees
// them in that order; returns the count, or -1 when the stack overflowed.
template <class F>
RD int mesh_query(const CmDesc& cm, v3 amin, v3 amax, F emit) {
    const v3 mn = V(amin.x * cm.inv_scale[0], amin.y * cm.inv_scale[1], amin.z * cm.inv_scale[2]);
    const v3 mx = V(amax.x * cm.inv_scale[0], amax.y * cm.inv_scale[1], amax.z * cm.inv_scale[2]);
    int stack[MESH_STACK];
    int sp = 0, count = 0;
    stack[sp++] = cm.root;
    while (sp > 0) {
        const int id = stack[--sp];
        if (id < 0) continue;
        const float4 lo = __ldg(&cm.nodes[id].lo), hi = __ldg(&cm.nodes[id].hi);
        // AABB::testCollision (AABB.h:179-187)
        if (mx.x < lo.x || hi.x < mn.x || mx.y < lo.y || hi.y < mn.y || mx.z < lo.z || hi.z < mn.z) continue;
        const int c0 = __float_as_int(lo.w);
        if (c0 <= -2) {
            emit(count, -2 - c0);
            count++;
        } else {
            if (sp + 2 > MESH_STACK) return -1;
            stack[sp++] = c0;
            stack[sp++] = __float_as_int(hi.w);
        }
    }
    return count;
}

__global__ void __launch_bounds__(128) hf_rects_kernel(const HfRectArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int4 it = a.items[i];
    v3 amin, amax;
    convex_aabb_in_concave(it, a.c_shape, a.shapes, a.bounds, a.c_wpos, a.c_wori, amin, amax);
    if (it.w & HF_MESH) {
        const int n = mesh_query(a.cm[it.z], amin, amax, [](int, int) {});
        if (n < 0) atomicOr(a.error, 2u);
        a.rect[i] = make_int4(0, n < 0 ? 0 : n, 0, 1);
        return;
    }
    const HfDesc hf = a.hf[it.z];
    // HeightFieldShape::computeOverlappingTriangles: the AABB without the scale
    const v3 inv = V(1.0f / hf.scale[0], 1.0f / hf.scale[1], 1.0f / hf.scale[2]);
    const float mn[3] = {amin.x * inv.x, amin.y * inv.y, amin.z * inv.z};
    const float mx[3] = {amax.x * inv.x, amax.y * inv.y, amax.z * inv.z};
    // computeMinMaxGridCoordinates: clamp into the bounds, shift to [0, extent],
    // round half up and widen by one cell (in double, as the reference's 0.5 literal)
    int minC[3], maxC[3];
    for (int k = 0; k < 3; k++) {
        float lo = fmax_std(mn[k], hf.bmin[k]);
        lo = fmin_std(lo, hf.bmax[k]);
        float hi = fmin_std(mx[k], hf.bmax[k]);
        hi = fmax_std(hi, hf.bmin[k]);
        const float tr = (hf.bmax[k] - hf.bmin[k]) * 0.5f;
        lo += tr;
        hi += tr;
        minC[k] = int(double(lo) + 0.5) - 1;
        maxC[k] = int(double(hi) + 0.5) + 1;
    }
    const int nc = int(hf.ncol) - 1, nr = int(hf.nrow) - 1;
    a.rect[i] = make_int4(clamp_int(minC[0], 0, nc), clamp_int(maxC[0], 0, nc), clamp_int(minC[2], 0, nr),
                          clamp_int(maxC[2], 0, nr));
}

// HeightField::getVertexAt (HeightField.cpp:388-398) times the shape's scale
RD v3 hf_vertex(const HfDesc& h, uint32_t x, uint32_t y) {
    const float height = __ldg(h.heights + size_t(y) * h.ncol + x);
    const v3 v = V(-h.width * 0.5f + float(x), h.origin + height, -h.length * 0.5f + float(y));
    return V(v.x * h.scale[0], v.y * h.scale[1], v.z * h.scale[2]);
}

__global__ void __launch_bounds__(128) hf_list_kernel(const HfListArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int4 it = a.items[i];
    if (!(it.w & HF_MESH)) return;
    v3 amin, amax;
    convex_aabb_in_concave(it, a.c_shape, a.shapes, a.bounds, a.c_wpos, a.c_wori, amin, amax);
    int32_t* out = a.tri_id + a.start[i];
    const uint32_t room = a.start[i + 1] - a.start[i];
    const int n = mesh_query(a.cm[it.z], amin, amax, [&](int k, int tri) {
        if (uint32_t(k) < room) out[k] = tri;
    });
    if (n < 0 || uint32_t(n) != room) atomicOr(a.error, 2u);
}

__global__ void __launch_bounds__(128) hf_tests_kernel(const HfTestArgs a) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n_tests) return;
    // the item holding test t: the last one whose first test is <= t
    uint32_t lo = 0, hi = a.n_items;  // start[lo] <= t < start[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.start[mid] <= t) lo = mid;
        else hi = mid;
    }
    const uint32_t ci = lo;
    const int4 it = a.items[ci];
    const int4 r = a.rect[ci];
    const uint32_t local = t - a.start[ci];
    const bool mesh = (it.w & HF_MESH) != 0;
    v3 v0, v1, v2, vn0, vn1, vn2;
    uint32_t i = 0, j = 0, k = 0;
    int32_t tri = -1;
    if (mesh) {
        // ConcaveMeshShape::getTriangleVertices / getTriangleVerticesNormals
        // (ConcaveMeshShape.cpp:79-104): scaled vertices, scaled vertex normals
        const CmDesc cm = a.cm[it.z];
        tri = a.tri_id[t];
        if (tri < 0 || uint32_t(tri) >= cm.nt) {
            atomicOr(a.error, 2u);
            tri = 0;
        }
        const uint32_t i0 = __ldg(cm.tris + 3 * tri), i1 = __ldg(cm.tris + 3 * tri + 1), i2 = __ldg(cm.tris + 3 * tri + 2);
        auto ld = [](const float* p, uint32_t v) { return V(__ldg(p + 3 * v), __ldg(p + 3 * v + 1), __ldg(p + 3 * v + 2)); };
        v0 = ld(cm.sverts, i0);
        v1 = ld(cm.sverts, i1);
        v2 = ld(cm.sverts, i2);
        vn0 = ld(cm.snormals, i0);
        vn1 = ld(cm.snormals, i1);
        vn2 = ld(cm.snormals, i2);
    } else {
        const uint32_t nj = uint32_t(r.w - r.z);
        const uint32_t cell = local >> 1;
        k = local & 1u;
        i = uint32_t(r.x) + cell / nj;
        j = uint32_t(r.z) + cell % nj;
        const HfDesc hf = a.hf[it.z];
        const v3 q1 = hf_vertex(hf, i, j), q2 = hf_vertex(hf, i, j + 1);
        const v3 q3 = hf_vertex(hf, i + 1, j), q4 = hf_vertex(hf, i + 1, j + 1);
        // first triangle (p1, p2, p3), second (p3, p2, p4); the vertex normals
        // are the face normal by getUnit()
        v0 = k == 0 ? q1 : q3;
        v1 = q2;
        v2 = k == 0 ? q3 : q4;
        vn0 = vn1 = vn2 = vunit(vcross(vsub(v1, v0), vsub(v2, v0)));
    }
    // TriangleShape's own normal (TriangleShape.cpp:40-60): normalize()
    const v3 fn = vnormalize(vcross(vsub(v1, v0), vsub(v2, v0)));
    const int4 b = a.batch[ci];
    const size_t n = size_t(b.y);
    float4* tr = a.tri + TRI_REC * size_t(b.x) + (t - uint32_t(b.x));
    tr[0] = make_float4(v0.x, v0.y, v0.z, 0.0f);
    tr[n] = make_float4(v1.x, v1.y, v1.z, 0.0f);
    tr[2 * n] = make_float4(v2.x, v2.y, v2.z, 0.0f);
    tr[3 * n] = make_float4(fn.x, fn.y, fn.z, 0.0f);
    tr[4 * n] = make_float4(vn0.x, vn0.y, vn0.z, 0.0f);
    tr[5 * n] = make_float4(vn1.x, vn1.y, vn1.z, 0.0f);
    tr[6 * n] = make_float4(vn2.x, vn2.y, vn2.z, 0.0f);
    const bool convex1 = (it.w & HF_SHAPE1_CONVEX) != 0;
    const int32_t sc = a.c_shape[it.x];
    const int row1 = convex1 ? it.x : it.y, row2 = convex1 ? it.y : it.x;
    a.s1[t] = convex1 ? sc : -1;
    a.s2[t] = convex1 ? -1 : sc;
    a.p1[t] = a.c_wpos[row1];
    a.r1[t] = a.c_wori[row1];
    a.p2[t] = a.c_wpos[row2];
    a.r2[t] = a.c_wori[row2];
    a.report[t] = (it.w & HF_NO_REPORT) ? 0 : 1;
    // the record of this triangle: kept from the previous step when the
    // triangle was tested then, else a new LastFrameCollisionInfo
    // (OverlappingPairs.h:86-91)
    const int32_t ps = a.prev_start[ci];
    const int4 pr = a.prev_rect[ci];
    int32_t pl = -1;
    if (ps >= 0 && mesh) {
        // the previous step's tests of this pair, in their query order
        for (int32_t q = 0; q < pr.y; q++)
            if (a.prev_tri_id[ps + q] == tri) {
                pl = q;
                break;
            }
    } else if (ps >= 0 && int(i) >= pr.x && int(i) < pr.y && int(j) >= pr.z && int(j) < pr.w) {
        pl = int32_t(((i - uint32_t(pr.x)) * uint32_t(pr.w - pr.z) + (j - uint32_t(pr.z))) * 2u + k);
    }
    if (pl >= 0) {
        a.cache[t] = a.prev_cache[uint32_t(ps) + uint32_t(pl)];
    } else {
        rp3dg_lastframe f;
        f.gjk_axis[0] = 0.0f;
        f.gjk_axis[1] = 1.0f;
        f.gjk_axis[2] = 0.0f;
        f.flags = 0;
        f.sat_face = 0;
        f.sat_edge1 = 0;
        f.sat_edge2 = 0;
        a.cache[t] = f;
    }
}

struct PotManifold {
    v3 n0;           // normal of its first point
    float largest;   // largest penetration depth of its points
    uint32_t count;
};

// shape-1 local points of one item's contacts: id = (test within item) * 16 + slot
struct ItemPoints {
    const float4* l1;
    uint32_t base;   // batch region start * 16
    uint32_t n;      // batch size
    uint32_t first;  // item's first test, relative to the batch
    RD v3 operator[](uint32_t id) const {
        const float4 p = l1[base + (id & 15u) * n + first + (id >> 4)];
        return V(p.x, p.y, p.z);
    }
};

__global__ void __launch_bounds__(128) hf_manifolds_kernel(const HfManifoldArgs a) {
    const uint32_t ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= a.n_items) return;
    const uint32_t st = a.start[ci], cnt = a.start[ci + 1] - st;
    const int4 b = a.batch[ci];
    const uint32_t base = uint32_t(b.x) * MAXC, bn = uint32_t(b.y), first = st - uint32_t(b.x);
    PotManifold pm[MAX_POTENTIAL_MANIFOLDS];
    uint32_t nman = 0;
    bool any = false;
    for (uint32_t u = 0; u < cnt; u++) {
        const uint32_t t = st + u;
        const bool col = a.is_colliding[t] != 0;
        // the record becomes valid and remembers whether the triangle collided
        uint8_t& f = a.cache[t].flags;
        f = uint8_t((f | RP3DG_LF_IS_VALID) & ~RP3DG_LF_WAS_COLLIDING) | (col ? RP3DG_LF_WAS_COLLIDING : 0);
        if (!col) continue;
        any = true;
        const uint32_t nbc = a.nb_contacts[t];
        for (uint32_t k = 0; k < nbc; k++) {
            const float4 nd = a.nd[base + k * bn + first + u];
            const v3 nrm = V(nd.x, nd.y, nd.z);
            uint32_t m = 255;
            for (uint32_t q = 0; q < nman; q++) {
                if (pm[q].count < MAX_POTENTIAL_POINTS && vdot(pm[q].n0, nrm) >= a.cos_similar) {
                    m = q;
                    break;
                }
            }
            if (m == 255 && nman < MAX_POTENTIAL_MANIFOLDS) {
                m = nman++;
                pm[m].n0 = nrm;
                pm[m].largest = 0.0f;
                pm[m].count = 0;
            }
            if (m != 255) {
                pm[m].count++;
                if (nd.w > pm[m].largest) pm[m].largest = nd.w;
            }
            a.mid[size_t(t) * MAXC + k] = uint8_t(m);
        }
    }
    // while more than NB_MAX_CONTACT_MANIFOLDS: drop the manifold whose deepest
    // point is the shallowest (first one on ties), replaced by the last one
    uint32_t order[MAX_POTENTIAL_MANIFOLDS];
    for (uint32_t q = 0; q < nman; q++) order[q] = q;
    uint32_t nm = nman;
    while (nm > HF_MAX_MANIFOLDS) {
        float minDepth = DECIMAL_LARGEST;
        uint32_t jmin = 0;
        for (uint32_t q = 0; q < nm; q++)
            if (pm[order[q]].largest < minDepth) {
                minDepth = pm[order[q]].largest;
                jmin = q;
            }
        order[jmin] = order[nm - 1];
        nm--;
    }
    const ItemPoints lp1{a.l1, base, bn, first};
    const int4 itm = a.items[ci];
    const float4 q4 = a.c_wori[(itm.w & HF_SHAPE1_CONVEX) ? itm.x : itm.y];
    const quat q1 = Q(q4.x, q4.y, q4.z, q4.w);
    uint32_t npts[HF_MAX_MANIFOLDS] = {0, 0, 0, 0};
    uint32_t idx[MAX_POTENTIAL_POINTS], cand[MAX_POTENTIAL_POINTS];
    for (uint32_t r = 0; r < nm; r++) {
        const uint32_t id = order[r];
        uint32_t nb = 0;
        for (uint32_t u = 0; u < cnt && nb < pm[id].count; u++) {
            const uint32_t t = st + u;
            if (!a.is_colliding[t]) continue;
            const uint32_t nbc = a.nb_contacts[t];
            for (uint32_t k = 0; k < nbc; k++)
                if (a.mid[size_t(t) * MAXC + k] == id) idx[nb++] = (u << 4) | k;
        }
        if (nb > 4) {
            const uint32_t p0 = idx[0];
            const float4 nd0 = a.nd[base + (p0 & 15u) * bn + first + (p0 >> 4)];
            reduce_points(idx, nb, lp1, V(nd0.x, nd0.y, nd0.z), q1, cand);
        }
        remove_duplicates(idx, nb, lp1);
        npts[r] = nb;
        for (uint32_t q = 0; q < nb; q++) {
            const uint32_t o = base + (idx[q] & 15u) * bn + first + (idx[q] >> 4);
            const size_t d = size_t(ci) * HF_OUT_POINTS + r * 4 + q;
            a.out_nd[d] = a.nd[o];
            a.out_l1[d] = a.l1[o];
            a.out_l2[d] = a.l2[o];
        }
    }
    a.out_coll[ci] = any ? 1 : 0;
    a.out_nman[ci] = uint8_t(nm);
    a.out_npts[ci] = make_uchar4(uint8_t(npts[0]), uint8_t(npts[1]), uint8_t(npts[2]), uint8_t(npts[3]));
}

}  // namespace

cudaError_t launch_hf_rects(const HfRectArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    hf_rects_kernel<<<(a.n + 127) / 128, 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_hf_list(const HfListArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    hf_list_kernel<<<(a.n + 127) / 128, 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_hf_tests(const HfTestArgs& a, cudaStream_t s) {
    if (a.n_tests == 0) return cudaSuccess;
    hf_tests_kernel<<<(a.n_tests + 127) / 128, 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_hf_manifolds(const HfManifoldArgs& a, cudaStream_t s) {
    if (a.n_items == 0) return cudaSuccess;
    hf_manifolds_kernel<<<(a.n_items + 127) / 128, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace rp3dg
