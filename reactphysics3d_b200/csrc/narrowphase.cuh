// Device restatement of ReactPhysics3D v0.10.2's six narrow-phase algorithms,
// one pair per thread.  Every floating-point expression keeps the reference's
// operation order (see rp3dg_math.cuh); control flow, early-outs, tolerances
// and the temporal-coherence cache behave as in the reference.  Paths below
// are inside the reference project.
#pragma once
#include "rp3dg_internal.h"
#include "rp3dg_math.cuh"
#include "../../include/rp3dg.h"

namespace rp3dg {

constexpr float REL_ERROR = 1.0e-3f;                     // GJKAlgorithm.h:44
constexpr float REL_ERROR_SQUARE = REL_ERROR * REL_ERROR;  // GJKAlgorithm.h:45
constexpr float SAT_REL_TOL = 1.002f;                    // SATAlgorithm.cpp:43
constexpr float SAT_ABS_TOL = 0.0005f;                   // SATAlgorithm.cpp:44
constexpr float SIMPLEX_EPS = 0.0001f;                   // VoronoiSimplex.cpp:33
constexpr uint32_t MAX_CONTACTS = RP3DG_MAX_CONTACTS_PER_PAIR;
constexpr uint32_t GJK_MAX_ITERATIONS = 1024;

struct hedge { uint32_t vertex, twin, face, next; };

// ---------------------------------------------------------------------------
// shapes
// ---------------------------------------------------------------------------
struct SphereS {
    float r;
    RD float margin() const { return r; }
    RD v3 support(v3) const { return V(0.0f, 0.0f, 0.0f); }  // SphereShape.h:149-153
};
struct CapsuleS {
    float r, hh;
    RD float margin() const { return r; }
    // CapsuleShape.h:191-206
    RD v3 support(v3 d) const {
        const float top = hh * d.y;
        const float bottom = -hh * d.y;
        if (top > bottom) return V(0.0f, hh, 0.0f);
        return V(0.0f, -hh, 0.0f);
    }
    // ConvexShape::getLocalSupportPointWithMargin (ConvexShape.cpp:40-56)
    RD v3 support_margin(v3 d) const {
        v3 sp = support(d);
        if (r != 0.0f) {
            v3 u = V(0.0f, -1.0f, 0.0f);
            if (vlen2(d) > MACHINE_EPSILON * MACHINE_EPSILON) u = vunit(d);
            sp = vadd(sp, vmul(u, r));
        }
        return sp;
    }
};

struct BoxPoly {
    v3 he;
    const BoxTables* t;
    RD float margin() const { return 0.0f; }
    RD uint32_t nfaces() const { return 6; }
    RD uint32_t nhe() const { return 24; }
    RD hedge edge(uint32_t e) const {
        const uint8_t* c = t->edges[e];
        hedge h; h.vertex = c[0]; h.twin = c[1]; h.face = c[2]; h.next = c[3];
        return h;
    }
    RD uint32_t face_edge(uint32_t f) const { return t->face_edge[f]; }
    RD uint32_t face_count(uint32_t) const { return 4; }
    RD uint32_t face_vertex(uint32_t f, uint32_t i) const { return t->face_verts[4 * f + i]; }
    // BoxShape::getVertexPosition (BoxShape.h:192-208): x positive for 1,2,5,6;
    // y positive for 2,3,6,7; z positive for 0..3
    RD v3 vertex(uint32_t v) const {
        return V(((0x66u >> v) & 1u) ? he.x : -he.x, ((0xCCu >> v) & 1u) ? he.y : -he.y,
                 ((0x0Fu >> v) & 1u) ? he.z : -he.z);
    }
    // BoxShape::getFaceNormal (BoxShape.h:211-225)
    RD v3 normal(uint32_t f) const {
        switch (f) {
            case 0: return V(0.0f, 0.0f, 1.0f);
            case 1: return V(1.0f, 0.0f, 0.0f);
            case 2: return V(0.0f, 0.0f, -1.0f);
            case 3: return V(-1.0f, 0.0f, 0.0f);
            case 4: return V(0.0f, -1.0f, 0.0f);
            default: return V(0.0f, 1.0f, 0.0f);
        }
    }
    RD v3 centroid() const { return V(0.0f, 0.0f, 0.0f); }
    // BoxShape::getLocalSupportPointWithoutMargin (BoxShape.h:166-171)
    RD v3 support(v3 d) const {
        return V(d.x < 0.0f ? -he.x : he.x, d.y < 0.0f ? -he.y : he.y, d.z < 0.0f ? -he.z : he.z);
    }
};

struct MeshPoly {
    const MeshHdr* h;
    const uint32_t* w;
    RD float margin() const { return 0.0f; }
    RD float f(uint32_t off) const { return __uint_as_float(w[off]); }
    RD uint32_t nfaces() const { return h->nf; }
    RD uint32_t nhe() const { return h->nhe; }
    RD hedge edge(uint32_t e) const {
        const uint32_t* c = w + h->off_edges + 4 * e;
        hedge r; r.vertex = c[0]; r.twin = c[1]; r.face = c[2]; r.next = c[3];
        return r;
    }
    RD uint32_t face_edge(uint32_t fi) const { return w[h->off_face_edge + fi]; }
    RD uint32_t face_count(uint32_t fi) const { return w[h->off_face_count + fi]; }
    RD uint32_t face_vertex(uint32_t fi, uint32_t i) const { return w[h->off_face_verts + w[h->off_face_start + fi] + i]; }
    // ConvexMeshShape::getVertexPosition (ConvexMeshShape.h:214-217), pre-scaled
    RD v3 vertex(uint32_t v) const { const uint32_t o = h->off_sverts + 3 * v; return V(f(o), f(o + 1), f(o + 2)); }
    // ConvexMeshShape::getFaceNormal (ConvexMeshShape.h:220-223)
    RD v3 normal(uint32_t fi) const { const uint32_t o = h->off_normals + 3 * fi; return V(f(o), f(o + 1), f(o + 2)); }
    RD v3 centroid() const { return V(h->centroid[0], h->centroid[1], h->centroid[2]); }
    // ConvexMeshShape::getLocalSupportPointWithoutMargin (ConvexMeshShape.cpp:80-102):
    // brute force over the unscaled vertices, strict '>' keeps the first maximum
    RD v3 support(v3 d) const {
        float maxd = DECIMAL_SMALLEST;
        uint32_t imax = 0;
        const uint32_t nv = h->nv;
        const uint32_t o = h->off_verts;
        for (uint32_t i = 0; i < nv; i++) {
            const float dp = vdot(d, V(f(o + 3 * i), f(o + 3 * i + 1), f(o + 3 * i + 2)));
            if (dp > maxd) { imax = i; maxd = dp; }
        }
        return vertex(imax);
    }
};

// TriangleShape (TriangleShape.h/.cpp): a two-faced convex polyhedron with
// margin 0; its topology is the shared triangle half-edge table.
struct TriPoly {
    v3 p0, p1, p2;       // mPoints
    v3 n;                // mNormal: cross product of the edges, normalize()d
    v3 vn0, vn1, vn2;    // mVerticesNormals
    const BoxTables* t;
    RD float margin() const { return 0.0f; }
    RD uint32_t nfaces() const { return 2; }
    RD uint32_t nhe() const { return 6; }
    RD hedge edge(uint32_t e) const {
        const uint8_t* c = t->tri_edges[e];
        hedge h; h.vertex = c[0]; h.twin = c[1]; h.face = c[2]; h.next = c[3];
        return h;
    }
    RD uint32_t face_edge(uint32_t f) const { return t->tri_face_edge[f]; }
    RD uint32_t face_count(uint32_t) const { return 3; }
    // faces (0, 1, 2) and (0, 2, 1)
    RD uint32_t face_vertex(uint32_t f, uint32_t i) const { return (f == 0 || i == 0) ? i : 3u - i; }
    RD v3 vertex(uint32_t v) const { return v == 0 ? p0 : (v == 1 ? p1 : p2); }
    // TriangleShape::getFaceNormal (TriangleShape.h:262-266)
    RD v3 normal(uint32_t f) const { return f == 0 ? n : vneg(n); }
    // TriangleShape::getCentroid (TriangleShape.h:269-271)
    RD v3 centroid() const { return vdivs(vadd(vadd(p0, p1), p2), 3.0f); }
    // TriangleShape::getLocalSupportPointWithoutMargin (TriangleShape.h:193-197) with
    // Vector3::getMaxAxis (Vector3.h:240-242)
    RD v3 support(v3 d) const {
        const float x = vdot(d, p0), y = vdot(d, p1), z = vdot(d, p2);
        const int k = x < y ? (y < z ? 2 : 1) : (x < z ? 2 : 0);
        return vertex(uint32_t(k));
    }
    // computeBarycentricCoordinatesInTriangle (mathematics_functions.h:203-219)
    // and computeSmoothLocalContactNormalForTriangle (TriangleShape.h:309-337)
    RD v3 smooth_normal(v3 p) const {
        const v3 e0 = vsub(p1, p0), e1 = vsub(p2, p0), e2 = vsub(p, p0);
        const float d00 = vdot(e0, e0), d01 = vdot(e0, e1), d11 = vdot(e1, e1);
        const float d20 = vdot(e2, e0), d21 = vdot(e2, e1);
        const float denom = d00 * d11 - d01 * d01;
        const float v = (d11 * d20 - d01 * d21) / denom;
        const float w = (d00 * d21 - d01 * d20) / denom;
        const float u = 1.0f - v - w;
        if (u > MACHINE_EPSILON && v > MACHINE_EPSILON && w > MACHINE_EPSILON) return n;
        const v3 in = vadd(vadd(vmul(vn0, u), vmul(vn1, v)), vmul(vn2, w));
        if (vlen2(in) < MACHINE_EPSILON) return n;
        return vunit(in);
    }
};

// ConvexPolyhedronShape::findMostAntiParallelFace (ConvexPolyhedronShape.h:105-123)
template <class P>
RD uint32_t most_antiparallel_face(const P& p, v3 dir) {
    float mind = DECIMAL_LARGEST;
    uint32_t best = 0;
    const uint32_t nf = p.nfaces();
    for (uint32_t i = 0; i < nf; i++) {
        const float d = vdot(p.normal(i), dir);
        if (d < mind) { mind = d; best = i; }
    }
    return best;
}

// ---------------------------------------------------------------------------
// per-pair state
// ---------------------------------------------------------------------------
struct LastFrame {
    v3 gjk_axis;
    uint32_t flags;
    uint32_t sat_face, sat_e1, sat_e2;
    RD bool has(uint32_t b) const { return (flags & b) != 0; }
    RD void set(uint32_t b, bool v) { flags = v ? (flags | b) : (flags & ~b); }
};

// Contact sink writing straight into the slot-major output arrays.
struct ContactSink {
    float4* nd;
    float4* l1;
    float4* l2;
    uint32_t n, i, max;
    uint32_t count;
    v3 first_normal;
    float first_depth;
    // NarrowPhaseInfoBatch::addContactPoint (NarrowPhaseInfoBatch.h:170-185)
    RD void add(v3 nrm, float depth, v3 p1, v3 p2, bool write = true) {
        if (count < MAX_CONTACTS) {
            if (count == 0) { first_normal = nrm; first_depth = depth; }
            if (write && count < max) {
                const size_t o = size_t(count) * n + i;
                nd[o] = make_float4(nrm.x, nrm.y, nrm.z, depth);
                l1[o] = make_float4(p1.x, p1.y, p1.z, 0.0f);
                l2[o] = make_float4(p2.x, p2.y, p2.z, 0.0f);
            }
            count++;
        }
    }
    RD void reset() { count = 0; }  // NarrowPhaseInfoBatch::resetContactPoints
};

struct Item {
    xform t1, t2;
    bool report;
    bool colliding;
    bool gjk_capped;
    uint32_t proposal;        // learned separating-feature class, 15 = none
    bool proposal_tested, proposal_confirmed;
    LastFrame lf;
    ContactSink out;
    uint32_t tri_side;        // 0: no triangle, 1: shape 1 is the triangle, 2: shape 2
    const TriPoly* tri;
#ifdef RP3DG_COUNT_EVENTS
    uint32_t ev[NP_EVENT_COUNT];  // path events of this pair (NpEvent)
#endif
};

// Path events: only the event-counting build (RP3DG_COUNT_EVENTS) keeps them;
// in the product build NP_EV expands to nothing and its arguments are never
// evaluated, so the timed kernels are unchanged.
#ifdef RP3DG_COUNT_EVENTS
#define NP_EV(it, e, k) ((it).ev[(e)] += uint32_t(k))
#define NP_EV_ONLY(...) __VA_ARGS__
#else
#define NP_EV(it, e, k) ((void)0)
#define NP_EV_ONLY(...)
#endif
// the support-point step of each shape kind, k times
RD void ev_support(Item& it, const SphereS&, uint32_t k = 1) { (void)it; (void)k; }
RD void ev_support(Item& it, const CapsuleS&, uint32_t k = 1) { (void)it; (void)k; NP_EV(it, EV_SUPPORT_CAPSULE, k); }
RD void ev_support(Item& it, const BoxPoly&, uint32_t k = 1) { (void)it; (void)k; NP_EV(it, EV_SUPPORT_BOX, k); }
RD void ev_support(Item& it, const MeshPoly& m, uint32_t k = 1) { (void)it; (void)m; (void)k; NP_EV(it, EV_SUPPORT_VERTEX, k * m.h->nv); }
RD void ev_support(Item& it, const TriPoly&, uint32_t k = 1) { (void)it; (void)k; NP_EV(it, EV_SUPPORT_TRI, k); }
// k face tests of testFacesDirectionPolyhedronVsPolyhedron against `other`
template <class P>
RD void ev_face_tests(Item& it, const P& other, uint32_t k) {
    NP_EV(it, EV_FACE_TEST, k);
    ev_support(it, other, k);
}

// TriangleShape::computeSmoothTriangleMeshContact (TriangleShape.h:342-365) and
// computeSmoothMeshContact (TriangleShape.cpp:90-115): the contact normal
// becomes the triangle's smooth normal at the contact point, oriented like the
// penetration axis, and the other shape's point is re-projected from it.
RD void smooth_triangle_contact(const Item& it, v3& nrm, float depth, v3& p1, v3& p2) {
    const bool tri1 = it.tri_side == 1;
    const v3 lpTri = tri1 ? p1 : p2;
    const xform triToWorld = tri1 ? it.t1 : it.t2;
    const xform worldToOther = tri1 ? xinv(it.t2) : xinv(it.t1);
    v3 ln = it.tri->smooth_normal(lpTri);
    v3 wn = qrot(triToWorld.q, ln);
    const v3 penAxis = tri1 ? nrm : vneg(nrm);
    if (vdot(wn, penAxis) < 0.0f) {
        wn = vneg(wn);
        ln = vneg(ln);
    }
    nrm = tri1 ? wn : vneg(wn);
    const v3 otherTri = vsub(lpTri, vmul(ln, depth));
    const v3 other = xapply(xmul(worldToOther, triToWorld), otherTri);
    if (tri1) p2 = other;
    else p1 = other;
}

// A contact of the GJK / SAT algorithms: smoothed first when one shape is a
// triangle (every addContactPoint of GJKAlgorithm.cpp and SATAlgorithm.cpp is
// preceded by computeSmoothTriangleMeshContact on the same arguments).
RD void emit(Item& it, v3& nrm, float depth, v3 p1, v3 p2, bool write = true) {
    if (it.tri_side) NP_EV(it, EV_TRI_SMOOTH, 1);
    if (it.tri_side) smooth_triangle_contact(it, nrm, depth, p1, p2);
    it.out.add(nrm, depth, p1, p2, write);
}

// ---------------------------------------------------------------------------
// SphereVsSphereAlgorithm::testCollision (SphereVsSphereAlgorithm.cpp:34-113)
// ---------------------------------------------------------------------------
RD void sphere_sphere(Item& it, float r1, float r2) {
    NP_EV(it, EV_CLOSED_FORM, 1);
    const xform t1 = it.t1, t2 = it.t2;
    const v3 d = vsub(t2.p, t1.p);
    const float d2 = vlen2(d);
    const float sum = r1 + r2;
    const float sum2 = sum * sum;
    if (d2 < sum2) {
        const float depth = sum - sqrtf(d2);
        if (depth > 0) {
            if (it.report) {
                const xform i1 = xinv(t1), i2 = xinv(t2);
                v3 p1, p2, n;
                if (d2 > MACHINE_EPSILON) {
                    p1 = vmul(vunit(xapply(i1, t2.p)), r1);
                    p2 = vmul(vunit(xapply(i2, t1.p)), r2);
                    n = vunit(d);
                } else {
                    n = V(0.0f, 1.0f, 0.0f);
                    p1 = vmul(qrot(i1.q, n), r1);
                    p2 = vmul(qrot(i2.q, n), r2);
                }
                NP_EV(it, EV_CLOSED_FORM_CONTACT, 1);
                it.out.add(n, depth, p1, p2);
            }
            it.colliding = true;
        }
    }
}

// SphereVsCapsuleAlgorithm::testCollision (SphereVsCapsuleAlgorithm.cpp:38-152)
RD void sphere_capsule(Item& it, bool sphere1, SphereS sph, CapsuleS cap) {
    NP_EV(it, EV_CLOSED_FORM, 1);
    const float capHeight = cap.hh + cap.hh;
    const float sr = sph.r, cr = cap.r;
    const xform s2w = sphere1 ? it.t1 : it.t2;
    const xform c2w = sphere1 ? it.t2 : it.t1;
    const xform s2c = xmul(xinv(c2w), s2w);
    const v3 center = s2c.p;
    const float half = capHeight * 0.5f;
    const v3 segA = V(0.0f, -half, 0.0f), segB = V(0.0f, half, 0.0f);
    const v3 closest = closest_point_on_segment(segA, segB, center);
    v3 c2s = vsub(closest, center);
    const float dist2 = vlen2(c2s);
    const float sum = sr + cr;
    if (dist2 < sum * sum) {
        if (it.report) {
            float depth;
            v3 nw, psph, pcap;
            if (dist2 > MACHINE_EPSILON) {
                const float dist = sqrtf(dist2);
                c2s = vdivs(c2s, dist);
                psph = xapply(xinv(s2c), vadd(center, vmul(c2s, sr)));
                pcap = vsub(closest, vmul(c2s, cr));
                nw = qrot(c2w.q, c2s);
                depth = sum - dist;
                if (!sphere1) nw = vneg(nw);
            } else {
                const v3 seg = vunit(vsub(segB, segA));
                const float cosA1 = fabsf(seg.x), cosA2 = fabsf(seg.y);
                depth = sum;
                const v3 ncap = cosA1 < cosA2 ? vcross(seg, V(1.0f, 0.0f, 0.0f)) : vcross(seg, V(0.0f, 1.0f, 0.0f));
                nw = qrot(c2w.q, ncap);
                psph = xapply(xinv(s2c), vadd(center, vmul(ncap, sr)));
                pcap = vsub(center, vmul(ncap, cr));
            }
            if (depth <= 0.0f) return;
            NP_EV(it, EV_CLOSED_FORM_CONTACT, 1);
            it.out.add(nw, depth, sphere1 ? psph : pcap, sphere1 ? pcap : psph);
        }
        it.colliding = true;
    }
}

// CapsuleVsCapsuleAlgorithm::testCollision (CapsuleVsCapsuleAlgorithm.cpp:37-243)
RD void capsule_capsule(Item& it, CapsuleS c1, CapsuleS c2) {
    NP_EV(it, EV_CLOSED_FORM, 1);
    const xform c1to2 = xmul(xinv(it.t2), it.t1);
    const float h1 = c1.hh + c1.hh, h2 = c2.hh + c2.hh;
    const float r1 = c1.r, r2 = c2.r;
    const float hh1 = h1 * 0.5f;
    const v3 s1a = xapply(c1to2, V(0.0f, -hh1, 0.0f));
    const v3 s1b = xapply(c1to2, V(0.0f, hh1, 0.0f));
    const float hh2 = h2 * 0.5f;
    const v3 s2a = V(0.0f, -hh2, 0.0f), s2b = V(0.0f, hh2, 0.0f);
    const v3 seg1 = vsub(s1b, s1a), seg2 = vsub(s2b, s2a);
    const float sum = r1 + r2;
    const bool parallel = are_parallel(seg1, seg2);
    if (parallel) {
        const float perp = point_to_line_distance(s1a, s1b, s2a);
        if (perp >= sum) return;
        const float d1 = vdot(seg1, s1a);
        const float d2 = -vdot(seg1, s1b);
        float t1 = plane_segment_intersection(s2b, s2a, d1, seg1);
        float t2 = plane_segment_intersection(s2a, s2b, d2, vneg(seg1));
        if (t1 > 0.0f && t2 > 0.0f) {
            if (it.report) {
                if (t1 > 1.0f) t1 = 1.0f;
                const v3 clipA = vsub(s2b, vmul(seg2, t1));
                if (t2 > 1.0f) t2 = 1.0f;
                const v3 clipB = vadd(s2a, vmul(seg2, t2));
                const v3 seg1n = vunit(seg1);
                const v3 onSeg1 = vadd(s1a, vmul(seg1n, vdot(seg1n, vsub(s2a, s1a))));
                v3 n2, s1to2;
                if (perp > MACHINE_EPSILON) {
                    s1to2 = vsub(s2a, onSeg1);
                    n2 = vunit(s1to2);
                } else {
                    const v3 seg2n = vunit(seg2);
                    const float cosA1 = fabsf(seg2n.x), cosA2 = fabsf(seg2n.y);
                    s1to2 = V(0.0f, 0.0f, 0.0f);
                    n2 = cosA1 < cosA2 ? vcross(seg2n, V(1.0f, 0.0f, 0.0f)) : vcross(seg2n, V(0.0f, 1.0f, 0.0f));
                }
                const xform c2to1 = xinv(c1to2);
                const v3 pA1 = xapply(c2to1, vadd(vsub(clipA, s1to2), vmul(n2, r1)));
                const v3 pB1 = xapply(c2to1, vadd(vsub(clipB, s1to2), vmul(n2, r1)));
                const v3 pA2 = vsub(clipA, vmul(n2, r2));
                const v3 pB2 = vsub(clipB, vmul(n2, r2));
                const float depth = sum - perp;
                const v3 nw = qrot(it.t2.q, n2);
                NP_EV(it, EV_CLOSED_FORM_CONTACT, 2);
                it.out.add(nw, depth, pA1, pA2);
                it.out.add(nw, depth, pB1, pB2);
            }
            it.colliding = true;
            return;
        }
    }
    v3 cp1, cp2;
    closest_points_segments(s1a, s1b, s2a, s2b, cp1, cp2);
    v3 d = vsub(cp2, cp1);
    const float dist2 = vlen2(d);
    if (dist2 < sum * sum) {
        if (it.report) {
            NP_EV(it, EV_CLOSED_FORM_CONTACT, 1);
            if (dist2 > MACHINE_EPSILON) {
                const float dist = sqrtf(dist2);
                d = vdivs(d, dist);
                const v3 p1 = xapply(xinv(c1to2), vadd(cp1, vmul(d, r1)));
                const v3 p2 = vsub(cp2, vmul(d, r2));
                it.out.add(qrot(it.t2.q, d), smax(sum - dist, MACHINE_EPSILON), p1, p2);
            } else if (parallel) {
                const float sq = vlen2(vsub(s1a, cp2));
                const v3 extreme = sq > MACHINE_EPSILON ? s1a : s1b;
                const v3 n2 = vnormalize(vsub(cp2, extreme));
                const v3 p1 = xapply(xinv(c1to2), vadd(cp1, vmul(n2, r1)));
                const v3 p2 = vsub(cp2, vmul(n2, r2));
                it.out.add(qrot(it.t2.q, n2), sum, p1, p2);
            } else {
                const v3 n2 = vnormalize(vcross(seg1, seg2));
                const v3 p1 = xapply(xinv(c1to2), vadd(cp1, vmul(n2, r1)));
                const v3 p2 = vsub(cp2, vmul(n2, r2));
                it.out.add(qrot(it.t2.q, n2), sum, p1, p2);
            }
        }
        it.colliding = true;
    }
}

// ---------------------------------------------------------------------------
// VoronoiSimplex (VoronoiSimplex.cpp:25-631)
// ---------------------------------------------------------------------------
struct Simplex {
    v3 pts[4], sa[4], sb[4];
    int n;
    float bary[4];
    bool recompute;
    v3 cp, cpa, cpb;
    bool valid;

    RD void init() { n = 0; recompute = false; valid = false; }
    RD void add(v3 p, v3 a, v3 b) { pts[n] = p; sa[n] = a; sb[n] = b; n++; recompute = true; }
    RD void remove(int i) { n--; pts[i] = pts[n]; sa[i] = sa[n]; sb[i] = sb[n]; }
    RD void reduce(int bits) {
        if (n >= 4 && (bits & 8) == 0) remove(3);
        if (n >= 3 && (bits & 4) == 0) remove(2);
        if (n >= 2 && (bits & 2) == 0) remove(1);
        if (n >= 1 && (bits & 1) == 0) remove(0);
    }
    RD bool contains(v3 p) const {
        for (int i = 0; i < n; i++) if (vlen2(vsub(pts[i], p)) <= SIMPLEX_EPS) return true;
        return false;
    }
    RD bool affinely_dependent() const {
        switch (n) {
            case 2: return vlen2(vsub(pts[1], pts[0])) <= SIMPLEX_EPS;
            case 3: return vlen2(vcross(vsub(pts[1], pts[0]), vsub(pts[2], pts[0]))) <= SIMPLEX_EPS;
            case 4: return fabsf(vdot(vsub(pts[1], pts[0]), vcross(vsub(pts[2], pts[0]), vsub(pts[3], pts[0])))) <= SIMPLEX_EPS;
        }
        return false;
    }
    RD void setbary(float a, float b, float c, float d) { bary[0] = a; bary[1] = b; bary[2] = c; bary[3] = d; }
    RD bool bary_valid() const { return bary[0] >= 0.0f && bary[1] >= 0.0f && bary[2] >= 0.0f && bary[3] >= 0.0f; }
    RD float max_len2() const {
        float m = 0.0f;
        for (int i = 0; i < n; i++) { const float l = vlen2(pts[i]); if (l > m) m = l; }
        return m;
    }
};

// computeClosestPointOnSegment (VoronoiSimplex.cpp:304-331)
RD void sx_seg(v3 a, v3 b, int& bits, float& t) {
    const v3 AP = vneg(a), AB = vsub(b, a);
    const float apab = vdot(AP, AB);
    if (apab > 0.0f) {
        const float l2 = vlen2(AB);
        if (apab < l2) { t = apab / l2; bits = 3; }
        else { t = 1.0f; bits = 2; }
    } else { t = 0.0f; bits = 1; }
}
// computeClosestPointOnTriangle (VoronoiSimplex.cpp:336-451)
RD void sx_tri(v3 a, v3 b, v3 c, int& bits, v3& bc) {
    const v3 ab = vsub(b, a), ac = vsub(c, a), ap = vneg(a);
    const float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { bc = V(1.0f, 0.0f, 0.0f); bits = 1; return; }
    const v3 bp = vneg(b);
    const float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { bc = V(0.0f, 1.0f, 0.0f); bits = 2; return; }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float v = d1 / (d1 - d3);
        bc = V(1.0f - v, v, 0.0f); bits = 3; return;
    }
    const v3 cp = vneg(c);
    const float d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { bc = V(0.0f, 0.0f, 1.0f); bits = 4; return; }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float w = d2 / (d2 - d6);
        bc = V(1.0f - w, 0.0f, w); bits = 5; return;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        bc = V(0.0f, 1.0f - w, w); bits = 6; return;
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    bc = V(1 - v - w, v, w);
    bits = 7;
}
// testOriginOutsideOfPlane (VoronoiSimplex.cpp:593-611)
RD int sx_outside(v3 a, v3 b, v3 c, v3 d) {
    const v3 nrm = vcross(vsub(b, a), vsub(c, a));
    const float signp = vdot(vneg(a), nrm);
    const float signd = vdot(vsub(d, a), nrm);
    if (signd * signd < SIMPLEX_EPS * SIMPLEX_EPS) return -1;
    return signp * signd < 0.0f;
}
RD int sx_map(int tri, int first, int second, int third) {
    return (((1 & tri) != 0) << first) | (((2 & tri) != 0) << second) | (((4 & tri) != 0) << third);
}
// computeClosestPointOnTetrahedron (VoronoiSimplex.cpp:456-575)
RD bool sx_tet(v3 a, v3 b, v3 c, v3 d, int& bits, float ab[2], float cd[2], bool& degenerate) {
    degenerate = false;
    bits = 15;
    ab[0] = ab[1] = cd[0] = cd[1] = 0.0f;
    const int oABC = sx_outside(a, b, c, d), oACD = sx_outside(a, c, d, b);
    const int oADB = sx_outside(a, d, b, c), oBDC = sx_outside(b, d, c, a);
    if (oABC < 0 || oACD < 0 || oADB < 0 || oBDC < 0) { degenerate = true; return false; }
    if (oABC == 0 && oACD == 0 && oADB == 0 && oBDC == 0) return true;
    float best = DECIMAL_LARGEST;
    int tb;
    v3 t;
    if (oABC) {
        sx_tri(a, b, c, tb, t);
        const float sd = vlen2(vadd(vadd(vmul(a, t.x), vmul(b, t.y)), vmul(c, t.z)));
        if (sd < best) { best = sd; ab[0] = t.x; ab[1] = t.y; cd[0] = t.z; cd[1] = 0.0f; bits = tb; }
    }
    if (oACD) {
        sx_tri(a, c, d, tb, t);
        const float sd = vlen2(vadd(vadd(vmul(a, t.x), vmul(c, t.y)), vmul(d, t.z)));
        if (sd < best) { best = sd; ab[0] = t.x; ab[1] = 0.0f; cd[0] = t.y; cd[1] = t.z; bits = sx_map(tb, 0, 2, 3); }
    }
    if (oADB) {
        sx_tri(a, d, b, tb, t);
        const float sd = vlen2(vadd(vadd(vmul(a, t.x), vmul(d, t.y)), vmul(b, t.z)));
        if (sd < best) { best = sd; ab[0] = t.x; ab[1] = t.z; cd[0] = 0.0f; cd[1] = t.y; bits = sx_map(tb, 0, 3, 1); }
    }
    if (oBDC) {
        sx_tri(b, d, c, tb, t);
        const float sd = vlen2(vadd(vadd(vmul(b, t.x), vmul(d, t.y)), vmul(c, t.z)));
        // the reference does not record the best distance for this last face
        if (sd < best) { ab[0] = 0.0f; ab[1] = t.x; cd[0] = t.z; cd[1] = t.y; bits = sx_map(tb, 1, 3, 2); }
    }
    return true;
}
// recomputeClosestPoint (VoronoiSimplex.cpp:169-299)
RD bool sx_recompute(Simplex& s) {
    if (s.recompute) {
        s.recompute = false;
        switch (s.n) {
            case 0: s.valid = false; break;
            case 1:
                s.cp = s.pts[0]; s.cpa = s.sa[0]; s.cpb = s.sb[0];
                s.setbary(1.0f, 0.0f, 0.0f, 0.0f);
                s.valid = s.bary_valid();
                break;
            case 2: {
                int bits = 0;
                float t;
                sx_seg(s.pts[0], s.pts[1], bits, t);
                s.cpa = vadd(s.sa[0], vmul(vsub(s.sa[1], s.sa[0]), t));
                s.cpb = vadd(s.sb[0], vmul(vsub(s.sb[1], s.sb[0]), t));
                s.cp = vsub(s.cpa, s.cpb);
                s.setbary(1.0f - t, t, 0.0f, 0.0f);
                s.valid = s.bary_valid();
                s.reduce(bits);
                break;
            }
            case 3: {
                int bits = 0;
                v3 bc;
                sx_tri(s.pts[0], s.pts[1], s.pts[2], bits, bc);
                s.cpa = vadd(vadd(vmul(s.sa[0], bc.x), vmul(s.sa[1], bc.y)), vmul(s.sa[2], bc.z));
                s.cpb = vadd(vadd(vmul(s.sb[0], bc.x), vmul(s.sb[1], bc.y)), vmul(s.sb[2], bc.z));
                s.cp = vsub(s.cpa, s.cpb);
                s.setbary(bc.x, bc.y, bc.z, 0.0f);
                s.valid = s.bary_valid();
                s.reduce(bits);
                break;
            }
            case 4: {
                int bits = 0;
                bool degenerate;
                float ab[2], cd[2];
                const bool outside = sx_tet(s.pts[0], s.pts[1], s.pts[2], s.pts[3], bits, ab, cd, degenerate);
                if (outside) {
                    s.cpa = vadd(vadd(vadd(vmul(s.sa[0], ab[0]), vmul(s.sa[1], ab[1])), vmul(s.sa[2], cd[0])), vmul(s.sa[3], cd[1]));
                    s.cpb = vadd(vadd(vadd(vmul(s.sb[0], ab[0]), vmul(s.sb[1], ab[1])), vmul(s.sb[2], cd[0])), vmul(s.sb[3], cd[1]));
                    s.cp = vsub(s.cpa, s.cpb);
                    s.setbary(ab[0], ab[1], cd[0], cd[1]);
                    s.reduce(bits);
                } else {
                    if (degenerate) {
                        s.valid = false;
                    } else {
                        s.setbary(0.0f, 0.0f, 0.0f, 0.0f);
                        s.cpa = V(0.0f, 0.0f, 0.0f); s.cpb = V(0.0f, 0.0f, 0.0f); s.cp = V(0.0f, 0.0f, 0.0f);
                        s.valid = true;
                    }
                    break;
                }
                s.valid = s.bary_valid();
                break;
            }
        }
    }
    return s.valid;
}

// ---------------------------------------------------------------------------
// GJKAlgorithm::testCollision (GJKAlgorithm.cpp:50-238)
// ---------------------------------------------------------------------------
enum GjkResult { GJK_SEPARATED = 0, GJK_COLLIDE_IN_MARGIN = 1, GJK_INTERPENETRATE = 2 };

template <class S1, class S2>
RD int gjk(Item& it, const S1& s1, const S2& s2) {
    NP_EV(it, EV_GJK_SETUP, 1);
    const xform t1 = it.t1, t2 = it.t2;
    const xform b2to1 = xmul(xinv(t1), t2);
    const quat rotToB2 = qmul(qinv(t2.q), t1.q);
    const float margin = s1.margin() + s2.margin();
    const float marginSquare = margin * margin;
    Simplex sx;
    sx.init();
    v3 v;
    if (it.lf.has(RP3DG_LF_IS_VALID) && it.lf.has(RP3DG_LF_WAS_USING_GJK)) v = it.lf.gjk_axis;
    else v = V(0.0f, 1.0f, 0.0f);
    float distSquare = DECIMAL_LARGEST;
    bool contactFound = false;
    uint32_t iterations = 0;
    do {
        // Safety bound only: the reference loop has no cap and converges in a
        // handful of iterations; a pair that reaches the bound is flagged.
        if (++iterations > GJK_MAX_ITERATIONS) { it.gjk_capped = true; contactFound = true; break; }
        NP_EV(it, EV_GJK_ITER, 1);
        ev_support(it, s1);
        ev_support(it, s2);
        const v3 suppA = s1.support(vneg(v));
        const v3 suppB = xapply(b2to1, s2.support(qrot(rotToB2, v)));
        const v3 w = vsub(suppA, suppB);
        const float vDotw = vdot(v, w);
        if (vDotw > 0.0f && vDotw * vDotw > distSquare * marginSquare) {
            it.lf.gjk_axis = v;
            return GJK_SEPARATED;
        }
        if (sx.contains(w) || distSquare - vDotw <= distSquare * REL_ERROR_SQUARE) { contactFound = true; break; }
        sx.add(w, suppA, suppB);
        if (sx.affinely_dependent()) { contactFound = true; break; }
        NP_EV(it, sx.n == 2 ? EV_SX_SEG : sx.n == 3 ? EV_SX_TRI : EV_SX_TET, sx.n >= 2 ? 1 : 0);
        const bool ok = sx_recompute(sx);
        v = sx.cp;
        if (!ok) { contactFound = true; break; }
        const float prevDistSquare = distSquare;
        distSquare = vlen2(v);
        if (prevDistSquare - distSquare <= MACHINE_EPSILON * prevDistSquare) {
            v = sx.cp;
            distSquare = vlen2(v);
            contactFound = true;
            break;
        }
    } while (sx.n != 4 && distSquare > MACHINE_EPSILON * sx.max_len2());

    if (contactFound && distSquare > MACHINE_EPSILON) {
        const float dist = sqrtf(distSquare);
        const v3 pA = vsub(sx.cpa, vmul(v, s1.margin() / dist));
        const v3 pB = xapply(xinv(b2to1), vadd(sx.cpb, vmul(v, s2.margin() / dist)));
        const v3 normal = qrot(t1.q, vneg(vunit(v)));
        const float depth = margin - dist;
        if (depth <= 0.0f) return GJK_SEPARATED;
        if (vlen2(normal) < MACHINE_EPSILON) return GJK_SEPARATED;
        NP_EV(it, EV_GJK_CONTACT, 1);
        if (it.report) {
            v3 nrm = normal;
            emit(it, nrm, depth, pA, pB);
        }
        return GJK_COLLIDE_IN_MARGIN;
    }
    return GJK_INTERPENETRATE;
}

// ---------------------------------------------------------------------------
// SAT (SATAlgorithm.cpp)
// ---------------------------------------------------------------------------

// testCollisionSphereVsConvexPolyhedron (SATAlgorithm.cpp:58-144) with
// computePolyhedronFaceVsSpherePenetrationDepth (:147-162)
template <class P>
RD void sat_sphere_poly(Item& it, bool sphere1, SphereS sph, const P& poly) {
    const xform s2w = sphere1 ? it.t1 : it.t2;
    const xform p2w = sphere1 ? it.t2 : it.t1;
    const xform s2p = xmul(xinv(p2w), s2w);
    const v3 center = s2p.p;
    float minDepth = DECIMAL_LARGEST;
    uint32_t minFace = 0;
    const uint32_t nf = poly.nfaces();
    for (uint32_t f = 0; f < nf; f++) {
        const v3 n = poly.normal(f);
        NP_EV(it, EV_SPHERE_FACE, 1);
        const float depth = vdot(vsub(poly.vertex(poly.face_vertex(f, 0)), center), n) + sph.r;
        if (depth <= 0.0f) return;
        if (depth < minDepth) { minDepth = depth; minFace = f; }
    }
    if (it.report) {
        NP_EV(it, EV_SPHERE_POLY_CONTACT, 1);
        const v3 mn = poly.normal(minFace);
        const v3 mnw = qrot(p2w.q, mn);
        const v3 psph = qrot(xinv(s2w).q, vmul(vneg(mnw), sph.r));
        const v3 ppoly = vadd(center, vmul(mn, minDepth - sph.r));
        v3 nw = sphere1 ? vneg(mnw) : mnw;
        emit(it, nw, minDepth, sphere1 ? psph : ppoly, sphere1 ? ppoly : psph);
    }
    it.colliding = true;
}

// computeCapsulePolyhedronFaceContactPoints (SATAlgorithm.cpp:381-470) with
// clipSegmentWithPlanes (mathematics_functions.h:256-326); the clip planes are
// generated edge by edge instead of being stored first (same arithmetic).
template <class P>
RD bool capsule_poly_face_contacts(uint32_t refFace, float capR, const P& poly, float depth, const xform& p2c,
                                   v3 nw, v3 sepAxisCap, v3 segAp, v3 segBp, Item& it, bool cap1) {
    const v3 fn = poly.normal(refFace);
    const uint32_t first = poly.face_edge(refFace);
    uint32_t e = first;
    v3 in0 = segAp, in1 = segBp;
    int nin = 2;
    v3 plane0 = V(0.0f, 0.0f, 0.0f);
    bool firstPlane = true;
    uint32_t guard = 0;  // a face cycle has at most MAX_FACE_VERTICES edges
    do {
        const hedge ed = poly.edge(e);
        const hedge tw = poly.edge(ed.twin);
        const v3 v1 = poly.vertex(ed.vertex);
        const v3 v2 = poly.vertex(tw.vertex);
        const v3 pn = vcross(fn, vsub(v2, v1));
        const v3 pp = poly.vertex(ed.vertex);
        NP_EV(it, EV_CAPSULE_CLIP, 1);
        if (firstPlane) { plane0 = pp; firstPlane = false; }
        if (nin != 0) {
            v3 o0 = V(0.0f, 0.0f, 0.0f), o1 = V(0.0f, 0.0f, 0.0f);
            int no = 0;
            const v3 a = in0, b = in1;
            const float an = vdot(vsub(a, pp), pn);
            const float bn = vdot(vsub(b, pp), pn);
            if (bn >= 0.0f) {
                if (an < 0.0f) {
                    const float t = plane_segment_intersection(a, b, vdot(pn, pp), pn);
                    o0 = (t >= 0.0f && t <= 1.0f) ? vadd(a, vmul(vsub(b, a), t)) : b;
                } else {
                    o0 = a;
                }
                o1 = b;
                no = 2;
            } else if (an >= 0.0f) {
                o0 = a;
                no = 1;
                const float t = plane_segment_intersection(a, b, -vdot(pn, pp), vneg(pn));
                if (t >= 0.0f && t <= 1.0f) {
                    o1 = vadd(a, vmul(vsub(b, a), t));
                    no = 2;
                } else {
                    // the segment is nearly parallel to the plane (t = -1): the
                    // reference keeps one vertex, and its next plane reads the
                    // array's second slot past its size, which still holds this
                    // plane's second vertex (Array::operator= clears and re-adds,
                    // Array.h:470-482): the segment goes on unchanged
                    o1 = b;
                }
            }
            in0 = o0; in1 = o1; nin = no;
        }
        e = ed.next;
    } while (e != first && ++guard < MAX_FACE_VERTICES);
    const v3 delta = vmul(fn, depth - capR);
    bool found = false;
    for (int i = 0; i < nin; i++) {
        const v3 c = i == 0 ? in0 : in1;
        const float cd = vdot(vsub(plane0, c), fn);
        if (cd > depth - capR - 0.001f) {
            if (!found) it.out.reset();
            found = true;
            const v3 pPoly = vadd(c, delta);
            const v3 pCap = vsub(xapply(p2c, c), vmul(sepAxisCap, capR));
            // normalWorld is a reference parameter there: a smoothed normal
            // carries into the next clipped point
            emit(it, nw, depth, cap1 ? pCap : pPoly, cap1 ? pPoly : pCap);
        }
    }
    return found;
}

// testCollisionCapsuleVsConvexPolyhedron (SATAlgorithm.cpp:165-319) with
// computePolyhedronFaceVsCapsulePenetrationDepth (:357-376),
// computeEdgeVsCapsuleInnerSegmentPenetrationDepth (:322-354) and
// isMinkowskiFaceCapsuleVsEdge (:476-482)
template <class P>
RD bool sat_capsule_poly(Item& it, bool cap1, CapsuleS cap, const P& poly) {
    const xform c2w = cap1 ? it.t1 : it.t2;
    const xform p2w = cap1 ? it.t2 : it.t1;
    const xform p2c = xmul(xinv(c2w), p2w);
    const float height = cap.hh + cap.hh;
    const v3 segA = V(0.0f, -height * 0.5f, 0.0f), segB = V(0.0f, height * 0.5f, 0.0f);
    const v3 segAxis = vsub(segB, segA);
    float minDepth = DECIMAL_LARGEST;
    uint32_t minFace = 0;
    bool isFace = false;
    v3 sepAxis = V(0.0f, 0.0f, 0.0f), sepE1 = V(0.0f, 0.0f, 0.0f), sepE2 = V(0.0f, 0.0f, 0.0f);
    const uint32_t nf = poly.nfaces();
    for (uint32_t f = 0; f < nf; f++) {
        const v3 fnc = qrot(p2c.q, poly.normal(f));
        NP_EV(it, EV_CAPSULE_FACE, 1);
        const v3 sp = cap.support_margin(vneg(fnc));
        const v3 pf = xapply(p2c, poly.vertex(poly.face_vertex(f, 0)));
        const float depth = vdot(vsub(pf, sp), fnc);
        if (depth <= 0.0f) return false;
        if (depth < minDepth) { minDepth = depth; minFace = f; isFace = true; sepAxis = fnc; }
    }
    const uint32_t nhe = poly.nhe();
    for (uint32_t e = 0; e < nhe; e += 2) {
        const hedge ed = poly.edge(e);
        const v3 ev1 = poly.vertex(ed.vertex);
        const v3 ev2 = poly.vertex(poly.edge(ed.next).vertex);
        const v3 edirc = qrot(p2c.q, vsub(ev2, ev1));
        const hedge tw = poly.edge(ed.twin);
        const v3 n1 = qrot(p2c.q, poly.normal(ed.face));
        const v3 n2 = qrot(p2c.q, poly.normal(tw.face));
        NP_EV(it, EV_CAPSULE_EDGE, 1);
        if (vdot(segAxis, n1) * vdot(segAxis, n2) < 0.0f) {
            NP_EV(it, EV_CAPSULE_EDGE_AXIS, 1);
            float depth = DECIMAL_LARGEST;
            v3 axis = vcross(segAxis, edirc);
            if (vlen2(axis) >= 0.00001f) {
                const v3 cen = xapply(p2c, poly.centroid());
                const v3 pe = xapply(p2c, ev1);
                if (vdot(axis, vsub(pe, cen)) < 0) axis = vneg(axis);
                axis = vnormalize(axis);
                const v3 sp = cap.support_margin(vneg(axis));
                depth = vdot(vsub(pe, sp), axis);
            }
            if (depth <= 0.0f) return false;
            if (depth < minDepth) { minDepth = depth; isFace = false; sepAxis = axis; sepE1 = ev1; sepE2 = ev2; }
        }
    }
    const xform c2p = xinv(p2c);
    const v3 segAp = xapply(c2p, segA), segBp = xapply(c2p, segB);
    v3 nw = qrot(c2w.q, sepAxis);
    if (cap1) nw = vneg(nw);
    if (isFace) {
        if (it.report) return capsule_poly_face_contacts(minFace, cap.r, poly, minDepth, p2c, nw, sepAxis, segAp, segBp, it, cap1);
    } else if (it.report) {
        v3 cpSeg, cpEdge;
        closest_points_segments(segAp, segBp, sepE1, sepE2, cpSeg, cpEdge);
        const v3 pCap = vsub(xapply(p2c, cpSeg), vmul(sepAxis, cap.r));
        emit(it, nw, minDepth, cap1 ? pCap : cpEdge, cap1 ? cpEdge : pCap);
    }
    return true;
}

// testSingleFaceDirectionPolyhedronVsPolyhedron (SATAlgorithm.cpp:1087-1110)
template <class P1, class P2>
RD float sat_single_face(const P1& p1, const P2& p2, const xform& p1to2, uint32_t f) {
    const v3 fn2 = qrot(p1to2.q, p1.normal(f));
    const v3 sp = p2.support(vneg(fn2));
    const v3 fv = xapply(p1to2, p1.vertex(p1.face_vertex(f, 0)));
    return vdot(vsub(fv, sp), fn2);
}
// testFacesDirectionPolyhedronVsPolyhedron (SATAlgorithm.cpp:1113-1142)
template <class P1, class P2>
RD float sat_faces(const P1& p1, const P2& p2, const xform& p1to2, uint32_t& minFace) {
    float minDepth = DECIMAL_LARGEST;
    const uint32_t nf = p1.nfaces();
    for (uint32_t f = 0; f < nf; f++) {
        const float d = sat_single_face(p1, p2, p1to2, f);
        if (d <= 0.0f) { minFace = f; return d; }
        if (d < minDepth) { minDepth = d; minFace = f; }
    }
    return minDepth;
}
// testGaussMapArcsIntersect (SATAlgorithm.cpp:1180-1191)
RD bool gauss_arcs(v3 a, v3 b, v3 c, v3 d, v3 bxa, v3 dxc) {
    const float cba = vdot(c, bxa), dba = vdot(d, bxa), adc = vdot(a, dxc), bdc = vdot(b, dxc);
    return cba * dba < 0.0f && adc * bdc < 0.0f && cba * bdc > 0.0f;
}
// The polyhedron-1 half of testEdgesBuildMinkowskiFace (SATAlgorithm.cpp:1146-1172):
// it only depends on edge 1, so it is evaluated once per edge of polyhedron 1.
struct Edge1Gauss { v3 a, b, bxa; };
template <class P1>
RD Edge1Gauss edge1_gauss(const P1& p1, const hedge& e1, const xform& p1to2) {
    Edge1Gauss g;
    g.a = qrot(p1to2.q, p1.normal(e1.face));
    const hedge tw = p1.edge(e1.twin);
    g.b = qrot(p1to2.q, p1.normal(tw.face));
    g.bxa = qrot(p1to2.q, vsub(p1.vertex(e1.vertex), p1.vertex(tw.vertex)));
    return g;
}
template <class P2>
RD bool edges_minkowski(const Edge1Gauss& g, const P2& p2, const hedge& e2) {
    const v3 c = p2.normal(e2.face);
    const hedge tw = p2.edge(e2.twin);
    const v3 d = p2.normal(tw.face);
    const v3 dxc = vsub(p2.vertex(e2.vertex), p2.vertex(tw.vertex));
    return gauss_arcs(g.a, g.b, vneg(c), vneg(d), g.bxa, dxc);
}
// The same test when polyhedron 2 is a box.  The box's face normals and edge
// vectors have one non-zero coordinate, so each of the four dot products of
// testGaussMapArcsIntersect equals one product (the other terms are signed
// zeros that cannot change a non-zero sum, and a zero result gives the same
// comparison outcome whatever its sign).  c and d are the negated normals, so
// c.bxa = -/+ bxa[m] exactly, and a.dxc = a[k] * D with D = +/-2h_k exactly.
RD float axis_component(v3 v, uint32_t axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
RD bool edges_minkowski(const Edge1Gauss& g, const BoxPoly& p2, const hedge& e2, uint32_t j) {
    const uint8_t* gi = p2.t->gauss[j];
    const uint32_t k = gi[0] & 3u, m = gi[1] & 3u, n = gi[2] & 3u;
    const float hk = axis_component(p2.he, k);
    const float D = (gi[0] & 4u) ? -(hk + hk) : (hk + hk);
    const float bm = axis_component(g.bxa, m), bn = axis_component(g.bxa, n);
    const float cba = (gi[1] & 4u) ? -bm : bm;
    const float dba = (gi[2] & 4u) ? -bn : bn;
    const float adc = axis_component(g.a, k) * D;
    const float bdc = axis_component(g.b, k) * D;
    (void)e2;
    return cba * dba < 0.0f && adc * bdc < 0.0f && cba * bdc > 0.0f;
}
template <class P2>
RD bool edges_minkowski(const Edge1Gauss& g, const P2& p2, const hedge& e2, uint32_t) {
    return edges_minkowski(g, p2, e2);
}

// computeDistanceBetweenEdges (SATAlgorithm.cpp:1040-1083): when shape 1 is a
// triangle the axis is oriented with shape 2's centroid c2 instead of c1
RD float sat_edge_distance(v3 e1A, v3 e2A, v3 c1, v3 d1, v3 d2, v3& outAxis, bool tri1 = false,
                           v3 c2 = V(0.0f, 0.0f, 0.0f)) {
    if (are_parallel(d1, d2)) return DECIMAL_LARGEST;
    v3 axis = vunit(vcross(d1, d2));
    const float dp = tri1 ? vdot(axis, vsub(e2A, c2)) : vdot(axis, vsub(c1, e1A));
    if (dp > 0.0f) axis = vneg(axis);
    outAxis = axis;
    return -vdot(axis, vsub(e2A, e1A));
}

// clipPolygonWithPlane (mathematics_functions.h:332-393)
RD uint32_t clip_polygon(const v3* in, uint32_t nin, v3 pp, v3 pn, v3* out, uint32_t* ninter = nullptr) {
    uint32_t no = 0;
    uint32_t vs = nin - 1;
    const float pnpp = vdot(pn, pp);
    float vsn = vdot(vsub(in[vs], pp), pn);
    for (uint32_t ve = 0; ve < nin; ve++) {
        const v3 a = in[vs], b = in[ve];
        const float ven = vdot(vsub(b, pp), pn);
        // writes are bounded by CLIP_MAX; a convex face never reaches it
        if (ven >= 0.0f) {
            if (vsn < 0.0f) {
                if (ninter) ++*ninter;
                const float t = plane_segment_intersection(a, b, pnpp, pn);
                if (no < CLIP_MAX) out[no++] = (t >= 0.0f && t <= 1.0f) ? vadd(a, vmul(vsub(b, a), t)) : b;
            }
            if (no < CLIP_MAX) out[no++] = b;
        } else if (vsn >= 0.0f) {
            if (ninter) ++*ninter;
            const float t = plane_segment_intersection(a, b, -pnpp, vneg(pn));
            if (no < CLIP_MAX) out[no++] = (t >= 0.0f && t <= 1.0f) ? vadd(a, vmul(vsub(b, a), t)) : a;
        }
        vs = ve;
        vsn = ven;
    }
    return no;
}

// computePolyhedronVsPolyhedronFaceContactPoints (SATAlgorithm.cpp:893-1036)
template <class PR, class PI>
RD bool face_contacts(bool ref1, const PR& refP, const PI& incP, const xform& r2i, const xform& i2r, uint32_t minFace,
                      Item& it) {
    const v3 axisR = refP.normal(minFace);
    const v3 axisI = qrot(r2i.q, axisR);
    const v3 nw = ref1 ? qrot(it.t1.q, axisR) : vneg(qrot(it.t2.q, axisR));
    const uint32_t incFace = most_antiparallel_face(incP, axisI);
    const uint32_t nInc = incP.face_count(incFace);
    NP_EV(it, EV_CLIP_SETUP, 1);
    NP_EV(it, EV_ANTIPARALLEL, incP.nfaces());
    NP_EV(it, EV_INC_VERTEX, nInc < CLIP_MAX ? nInc : CLIP_MAX);
    NP_EV_ONLY(uint32_t ninter = 0;)
    v3 buf1[CLIP_MAX], buf2[CLIP_MAX];
    uint32_t n1 = 0, n2 = 0;
    for (uint32_t i = 0; i < nInc && i < CLIP_MAX; i++) buf1[n1++] = xapply(i2r, incP.vertex(incP.face_vertex(incFace, i)));
    const uint32_t firstEdge = refP.face_edge(minFace);
    bool v1in = false;
    uint32_t nOut = 0, curIdx, guard = 0;
    hedge cur = refP.edge(firstEdge);
    v3 ev1 = refP.vertex(cur.vertex);
    do {
        v1in = !v1in;
        const hedge nxt = refP.edge(cur.next);
        const v3 ev2 = refP.vertex(nxt.vertex);
        const v3 pn = vcross(axisR, vsub(ev2, ev1));
        NP_EV(it, EV_CLIP_PLANE, 1);
        NP_EV(it, EV_CLIP_VERTEX, v1in ? n1 : n2);
#ifdef RP3DG_COUNT_EVENTS
        if (v1in) n2 = clip_polygon(buf1, n1, ev1, pn, buf2, &ninter);
        else n1 = clip_polygon(buf2, n2, ev1, pn, buf1, &ninter);
#else
        if (v1in) n2 = clip_polygon(buf1, n1, ev1, pn, buf2);
        else n1 = clip_polygon(buf2, n2, ev1, pn, buf1);
#endif
        curIdx = cur.next;
        cur = nxt;
        ev1 = ev2;
        if (v1in) { n1 = 0; nOut = n2; }
        else { n2 = 0; nOut = n1; }
    } while (curIdx != firstEdge && nOut > 0 && ++guard < MAX_FACE_VERTICES);
    const v3* clipped = v1in ? buf2 : buf1;
    const uint32_t nClip = v1in ? n2 : n1;
    const v3 refV = refP.vertex(refP.edge(firstEdge).vertex);
    bool found = false;
    NP_EV(it, EV_CLIP_INTERSECT, ninter);
    NP_EV(it, EV_CLIP_DEPTH, nClip);
    for (uint32_t i = 0; i < nClip; i++) {
        const float depth = vdot(vsub(refV, clipped[i]), axisR);
        if (depth > 0.0f) {
            found = true;
            if (it.report) {
                NP_EV(it, EV_CONTACT, 1);
                const v3 pInc = xapply(r2i, clipped[i]);
                const v3 pRef = project_onto_plane(clipped[i], axisR, refV);
                v3 onw = nw;  // outWorldNormal: a copy per clipped point
                emit(it, onw, depth, ref1 ? pRef : pInc, ref1 ? pInc : pRef);
            }
        }
    }
    return found;
}

template <class P1, class P2>
RD bool poly_face_contacts(bool ref1, const P1& p1, const P2& p2, const xform& p1to2, const xform& p2to1, uint32_t minFace,
                           Item& it) {
    if (ref1) return face_contacts(true, p1, p2, p1to2, p2to1, minFace, it);
    return face_contacts(false, p2, p1, p2to1, p1to2, minFace, it);
}

template <class P> struct IsBox { static constexpr bool value = false; };
template <> struct IsBox<BoxPoly> { static constexpr bool value = true; };
template <class P> struct IsTri { static constexpr bool value = false; };
template <> struct IsTri<TriPoly> { static constexpr bool value = true; };
RD const BoxTables* box_tables_of(const BoxPoly& b, const BoxPoly&) { return b.t; }
RD const BoxTables* box_tables_of(const BoxPoly& b, const MeshPoly&) { return b.t; }
RD const BoxTables* box_tables_of(const MeshPoly&, const BoxPoly& b) { return b.t; }
RD const BoxTables* box_tables_of(const MeshPoly&, const MeshPoly&) { return nullptr; }
template <class P1, class P2>
RD const BoxTables* box_tables_of(const P1&, const P2&) { return nullptr; }

// ---------------------------------------------------------------------------
// exact confirmation of a proposed feature
// ---------------------------------------------------------------------------
// Tests the proposed feature with the reference's own arithmetic; on a
// separating axis fills the cache like the reference's full SAT would for
// that feature and returns true.
template <class P1, class P2>
RD bool confirm_proposal(uint32_t cls, const P1& p1, const P2& p2, const xform& p1to2, const xform& p2to1,
                         LastFrame& lf, bool box1, bool box2, const BoxTables* bt) {
    if (cls < 3) {
        if (!box1) return false;
        const uint32_t fp = cls == 0 ? 1u : (cls == 1 ? 5u : 0u), fm = cls == 0 ? 3u : (cls == 1 ? 4u : 2u);
        for (int s = 0; s < 2; s++) {
            const uint32_t f = s == 0 ? fp : fm;
            if (sat_single_face(p1, p2, p1to2, f) <= 0.0f) {
                lf.set(RP3DG_LF_SAT_FACE_POLY1, true); lf.set(RP3DG_LF_SAT_FACE_POLY2, false); lf.sat_face = f;
                return true;
            }
        }
        return false;
    }
    if (cls < 6) {
        if (!box2) return false;
        const uint32_t c = cls - 3;
        const uint32_t fp = c == 0 ? 1u : (c == 1 ? 5u : 0u), fm = c == 0 ? 3u : (c == 1 ? 4u : 2u);
        for (int s = 0; s < 2; s++) {
            const uint32_t f = s == 0 ? fp : fm;
            if (sat_single_face(p2, p1, p2to1, f) <= 0.0f) {
                lf.set(RP3DG_LF_SAT_FACE_POLY1, false); lf.set(RP3DG_LF_SAT_FACE_POLY2, true); lf.sat_face = f;
                return true;
            }
        }
        return false;
    }
    if (cls < 15 && box1 && box2) {
        const uint32_t a = (cls - 6) / 3, b = (cls - 6) % 3;
        const v3 c1 = xapply(p1to2, p1.centroid());
        for (int ii = 0; ii < 4; ii++) {
            const uint32_t i = bt->axis_edges[a][ii];
            const hedge e1 = p1.edge(i);
            const v3 e1A = xapply(p1to2, p1.vertex(e1.vertex));
            const v3 e1B = xapply(p1to2, p1.vertex(p1.edge(e1.next).vertex));
            const Edge1Gauss g = edge1_gauss(p1, e1, p1to2);
            for (int jj = 0; jj < 4; jj++) {
                const uint32_t j = bt->axis_edges[b][jj];
                const hedge e2 = p2.edge(j);
                if (edges_minkowski(g, p2, e2, j)) {
                    const v3 e2A = p2.vertex(e2.vertex);
                    const v3 e2B = p2.vertex(p2.edge(e2.next).vertex);
                    v3 axis;
                    const float d = sat_edge_distance(e1A, e2A, c1, vsub(e1B, e1A), vsub(e2B, e2A), axis);
                    if (d <= 0.0f) {
                        lf.set(RP3DG_LF_SAT_FACE_POLY1, false); lf.set(RP3DG_LF_SAT_FACE_POLY2, false);
                        lf.sat_e1 = i; lf.sat_e2 = j;
                        return true;
                    }
                }
            }
        }
    }
    return false;
}

// testCollisionConvexPolyhedronVsConvexPolyhedron (SATAlgorithm.cpp:485-889)
template <class P1, class P2>
RD void sat_poly_poly(Item& it, const P1& p1, const P2& p2, bool clipPrev) {
    NP_EV(it, EV_POLY_SETUP, 1);
    const xform p1to2 = xmul(xinv(it.t2), it.t1);
    const xform p2to1 = xinv(p1to2);
    LastFrame& lf = it.lf;

    // A cache naming a face or half-edge the shapes do not have cannot come
    // from a previous frame of this pair; it is ignored instead of indexed.
    const bool cacheInRange = lf.has(RP3DG_LF_SAT_FACE_POLY1)   ? lf.sat_face < p1.nfaces()
                              : lf.has(RP3DG_LF_SAT_FACE_POLY2) ? lf.sat_face < p2.nfaces()
                                                                : (lf.sat_e1 < p1.nhe() && lf.sat_e2 < p2.nhe());
    if (cacheInRange && lf.has(RP3DG_LF_IS_VALID) && lf.has(RP3DG_LF_WAS_USING_SAT)) {
        const bool wasColliding = lf.has(RP3DG_LF_WAS_COLLIDING);
        if (lf.has(RP3DG_LF_SAT_FACE_POLY1) || lf.has(RP3DG_LF_SAT_FACE_POLY2)) {
            const bool face1 = lf.has(RP3DG_LF_SAT_FACE_POLY1);
            const float d = face1 ? sat_single_face(p1, p2, p1to2, lf.sat_face) : sat_single_face(p2, p1, p2to1, lf.sat_face);
            if (face1) ev_face_tests(it, p2, 1);
            else ev_face_tests(it, p1, 1);
            if (!wasColliding && d <= 0.0f) return;
            if (wasColliding && clipPrev && d > 0.0f) {
                if (poly_face_contacts(face1, p1, p2, p1to2, p2to1, lf.sat_face, it)) {
                    lf.set(RP3DG_LF_SAT_FACE_POLY1, face1);
                    lf.set(RP3DG_LF_SAT_FACE_POLY2, !face1);
                    it.colliding = true;
                    return;
                }
            }
        } else {
            const hedge e1 = p1.edge(lf.sat_e1);
            const hedge e2 = p2.edge(lf.sat_e2);
            const v3 e1A = xapply(p1to2, p1.vertex(e1.vertex));
            const v3 e1B = xapply(p1to2, p1.vertex(p1.edge(e1.next).vertex));
            const v3 d1 = vsub(e1B, e1A);
            const v3 e2A = p2.vertex(e2.vertex);
            const v3 e2B = p2.vertex(p2.edge(e2.next).vertex);
            const v3 d2 = vsub(e2B, e2A);
            NP_EV(it, EV_EDGE1, 1);
            NP_EV(it, EV_GAUSS, 1);
            if (edges_minkowski(edge1_gauss(p1, e1, p1to2), p2, e2, lf.sat_e2)) {
                NP_EV(it, EV_EDGE_DIST, 1);
                v3 axis;
                const v3 c1 = xapply(p1to2, p1.centroid());
                const float d = sat_edge_distance(e1A, e2A, c1, d1, d2, axis, IsTri<P1>::value,
                                                  IsTri<P1>::value ? p2.centroid() : V(0.0f, 0.0f, 0.0f));
                if (!wasColliding && d <= 0.0f) return;
                if (wasColliding && clipPrev && d > 0.0f && d < DECIMAL_LARGEST) {
                    v3 cp1, cp2;
                    closest_points_segments(e1A, e1B, e2A, e2B, cp1, cp2);
                    const float l1 = vlen2(d1), l2 = vlen2(d2);
                    const float t1 = vdot(vsub(cp1, e2A), d2) / l2;
                    const float t2 = vdot(vsub(cp2, e1A), d1) / l1;
                    NP_EV(it, EV_EDGE_CONTACT, 1);
                    if (t1 >= 0.0f && t1 <= 1.0f && t2 >= 0.0f && t2 <= 1.0f) {
                        if (it.report) {
                            v3 nw = qrot(it.t2.q, axis);
                            emit(it, nw, d, xapply(p2to1, cp1), cp2);
                        }
                        it.colliding = true;
                        return;
                    }
                }
            }
        }
    }

    // learned proposal: tested where the reference starts its full SAT
    if (it.proposal < 15) {
        it.proposal_tested = true;
        if (confirm_proposal(it.proposal, p1, p2, p1to2, p2to1, lf, IsBox<P1>::value, IsBox<P2>::value, box_tables_of(p1, p2))) {
            it.proposal_confirmed = true;
            return;
        }
    }
    float minDepth;
    uint32_t minFace;
    bool isFace1;
    uint32_t f1 = 0, f2 = 0;
    const float d1 = sat_faces(p1, p2, p1to2, f1);
    ev_face_tests(it, p2, d1 <= 0.0f ? f1 + 1 : p1.nfaces());
    if (d1 <= 0.0f) {
        lf.set(RP3DG_LF_SAT_FACE_POLY1, true); lf.set(RP3DG_LF_SAT_FACE_POLY2, false); lf.sat_face = f1;
        return;
    }
    const float d2 = sat_faces(p2, p1, p2to1, f2);
    ev_face_tests(it, p1, d2 <= 0.0f ? f2 + 1 : p2.nfaces());
    if (d2 <= 0.0f) {
        lf.set(RP3DG_LF_SAT_FACE_POLY1, false); lf.set(RP3DG_LF_SAT_FACE_POLY2, true); lf.sat_face = f2;
        return;
    }
    bool isFace = true;
    minDepth = smin(d1, d2);
    if (d1 < d2 * SAT_REL_TOL + SAT_ABS_TOL) { minFace = f1; isFace1 = true; }
    else { minFace = f2; isFace1 = false; }

    uint32_t minE1 = 0, minE2 = 0;
    v3 sE1A = V(0.0f, 0.0f, 0.0f), sE1B = sE1A, sE2A = sE1A, sE2B = sE1A, minEdgeAxis = sE1A;
    const v3 c1 = xapply(p1to2, p1.centroid());
    const uint32_t nhe1 = p1.nhe(), nhe2 = p2.nhe();
    for (uint32_t i = 0; i < nhe1; i += 2) {
        const hedge e1 = p1.edge(i);
        const v3 e1A = xapply(p1to2, p1.vertex(e1.vertex));
        const v3 e1B = xapply(p1to2, p1.vertex(p1.edge(e1.next).vertex));
        const v3 dir1 = vsub(e1B, e1A);
        const Edge1Gauss g = edge1_gauss(p1, e1, p1to2);
        NP_EV(it, EV_EDGE1, 1);
        for (uint32_t j = 0; j < nhe2; j += 2) {
            const hedge e2 = p2.edge(j);
            NP_EV(it, EV_GAUSS, 1);
            if (edges_minkowski(g, p2, e2, j)) {
                NP_EV(it, EV_EDGE_DIST, 1);
                const v3 e2A = p2.vertex(e2.vertex);
                const v3 e2B = p2.vertex(p2.edge(e2.next).vertex);
                v3 axis;
                const float d = sat_edge_distance(e1A, e2A, c1, dir1, vsub(e2B, e2A), axis, IsTri<P1>::value,
                                                  IsTri<P1>::value ? p2.centroid() : V(0.0f, 0.0f, 0.0f));
                if (d <= 0.0f) {
                    lf.set(RP3DG_LF_SAT_FACE_POLY1, false); lf.set(RP3DG_LF_SAT_FACE_POLY2, false);
                    lf.sat_e1 = i; lf.sat_e2 = j;
                    return;
                }
                if ((isFace && d * SAT_REL_TOL + SAT_ABS_TOL < minDepth) || (!isFace && d < minDepth)) {
                    minDepth = d; isFace1 = false; isFace = false; minE1 = i; minE2 = j;
                    sE1A = e1A; sE1B = e1B; sE2A = e2A; sE2B = e2B; minEdgeAxis = axis;
                }
            }
        }
    }
    if (isFace) {
        const bool found = poly_face_contacts(isFace1, p1, p2, p1to2, p2to1, minFace, it);
        lf.set(RP3DG_LF_SAT_FACE_POLY1, isFace1); lf.set(RP3DG_LF_SAT_FACE_POLY2, !isFace1); lf.sat_face = minFace;
        if (!found) return;
    } else {
        if (it.report) {
            NP_EV(it, EV_EDGE_CONTACT, 1);
            v3 cp1, cp2;
            closest_points_segments(sE1A, sE1B, sE2A, sE2B, cp1, cp2);
            v3 nw = qrot(it.t2.q, minEdgeAxis);
            emit(it, nw, minDepth, xapply(p2to1, cp1), cp2);
        }
        lf.set(RP3DG_LF_SAT_FACE_POLY1, false); lf.set(RP3DG_LF_SAT_FACE_POLY2, false);
        lf.sat_e1 = minE1; lf.sat_e2 = minE2;
    }
    it.colliding = true;
}

// ---------------------------------------------------------------------------
// algorithm wrappers
// ---------------------------------------------------------------------------

// SphereVsConvexPolyhedronAlgorithm::testCollision (SphereVsConvexPolyhedronAlgorithm.cpp:38-103)
template <class P>
RD void sphere_poly(Item& it, bool sphere1, SphereS s, const P& poly) {
    const int r = sphere1 ? gjk(it, s, poly) : gjk(it, poly, s);
    it.lf.set(RP3DG_LF_WAS_USING_GJK, true); it.lf.set(RP3DG_LF_WAS_USING_SAT, false);
    if (r == GJK_COLLIDE_IN_MARGIN) { it.colliding = true; return; }
    if (r == GJK_INTERPENETRATE) {
        sat_sphere_poly(it, sphere1, s, poly);
        it.lf.set(RP3DG_LF_WAS_USING_GJK, false); it.lf.set(RP3DG_LF_WAS_USING_SAT, true);
    }
}

// CapsuleVsConvexPolyhedronAlgorithm::testCollision (CapsuleVsConvexPolyhedronAlgorithm.cpp:42-177)
template <class P>
RD void capsule_poly(Item& it, bool cap1, CapsuleS cap, const P& poly) {
    const int r = cap1 ? gjk(it, cap, poly) : gjk(it, poly, cap);
    it.lf.set(RP3DG_LF_WAS_USING_GJK, true); it.lf.set(RP3DG_LF_WAS_USING_SAT, false);
    if (r == GJK_COLLIDE_IN_MARGIN) {
        if (it.report) {
            // contactPoint refers to the GJK contact (slot 0); it only changes
            // when contacts are found, after which the loop stops
            const v3 cn = it.out.first_normal;
            const float cdepth = it.out.first_depth;
            const xform p2w = cap1 ? it.t2 : it.t1;
            const xform c2w = cap1 ? it.t1 : it.t2;
            const float h = cap.hh + cap.hh;
            const v3 segA = V(0.0f, -h * 0.5f, 0.0f), segB = V(0.0f, h * 0.5f, 0.0f);
            const v3 segDir = vnormalize(qrot(c2w.q, vsub(segB, segA)));
            const uint32_t nf = poly.nfaces();
            for (uint32_t f = 0; f < nf; f++) {
                const v3 fn = poly.normal(f);
                NP_EV(it, EV_CAPSULE_GJK_FACE, 1);
                v3 fnw = qrot(p2w.q, fn);
                const bool inDir = vdot(fnw, cn) > 0.0f;
                const bool inContactDir = (cap1 && !inDir) || (!cap1 && inDir);
                if (inContactDir && are_orthogonal(fnw, segDir) && are_parallel(fnw, cn)) {
                    const xform p2c = xmul(xinv(c2w), p2w);
                    const xform c2p = xinv(p2c);
                    const v3 segAp = xapply(c2p, segA), segBp = xapply(c2p, segB);
                    const v3 sepAxisCap = qrot(p2c.q, fn);
                    if (cap1) fnw = vneg(fnw);
                    if (capsule_poly_face_contacts(f, cap.r, poly, cdepth, p2c, fnw, sepAxisCap, segAp, segBp, it, cap1)) break;
                }
            }
        }
        it.colliding = true;
        return;
    }
    if (r == GJK_INTERPENETRATE) {
        it.colliding = sat_capsule_poly(it, cap1, cap, poly);
        it.lf.set(RP3DG_LF_WAS_USING_GJK, false); it.lf.set(RP3DG_LF_WAS_USING_SAT, true);
    }
}


// ===========================================================================
// Warp-cooperative SAT for two convex polyhedra: one warp per pair.
//
// The reference visits faces and edge pairs one after another and keeps
// (a) the first candidate axis (in visiting order) that separates the shapes
// and (b) otherwise the minimum penetration depth, first occurrence on ties.
// Here the 32 lanes evaluate 32 consecutive candidates at a time with the
// reference's per-candidate arithmetic, then
//   - a ballot over "separates" in visiting order finds the same first
//     separating candidate (earlier groups had none), and
//   - an (depth, index) arg-min with the smaller index winning ties gives
//     the same minimum and the same index.
// For the edge pairs the reference biases the comparison against the face
// minimum: an edge pair k only takes over if fl(fl(d_k*1.002)+0.0005) <
// faceMin, after which later pairs need only d < current minimum.  Because
// rounding is monotonic, every pair before the first qualifying k has a
// larger depth than d_k, so the final choice is the global first arg-min,
// taken exactly when that minimum itself qualifies.  Results are therefore
// bit-identical to the sequential loops.
// ===========================================================================
constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr uint32_t WARP_EDGE_CAP = 128;  // even half-edges of polyhedron 1 staged per warp

// Optional per-phase cycle counters (the device counterpart of the
// reference's RP3D_PROFILE scopes), compiled in with -DRP3DG_PROFILE_PHASES.
#ifdef RP3DG_PROFILE_PHASES
__device__ unsigned long long g_phase_cycles[8];
__device__ unsigned long long g_phase_count[8];
struct PhaseTimer {
    long long t;
    int lane;
    RD PhaseTimer(int l) : t(0), lane(l) {
#ifdef __CUDA_ARCH__
        t = clock64();
#endif
    }
    RD void mark(int phase) {
#ifdef __CUDA_ARCH__
        const long long now = clock64();
        if (lane == 0) { atomicAdd(&g_phase_cycles[phase], (unsigned long long)(now - t)); atomicAdd(&g_phase_count[phase], 1ull); }
        t = now;
#endif
    }
};
#else
struct PhaseTimer {
    RD PhaseTimer(int) {}
    RD void mark(int) {}
};
#endif

// Per-edge data of polyhedron 1 in polyhedron-2 space, staged in shared memory.
struct Edge1Stage {
    float e1A[3], dir1[3], a[3], b[3], bxa[3];
};
// Shared-memory scratch of one warp: staged edges, the list of edge pairs
// that pass the Gauss-map test (in visiting order) and the clip polygon.
constexpr uint32_t WARP_CAND_CAP = 512;
struct WarpScratch {
    union {
        Edge1Stage stage[WARP_EDGE_CAP];
        float feat[32][32];  // a tile's MLP input rows (consumed before the SAT starts)
    };
    uint16_t cand[WARP_CAND_CAP];
    v3 poly[CLIP_MAX];
    uint32_t cls[32];
};

RD void warp_argmin(float& d, uint32_t& idx) {
    for (int o = 16; o; o >>= 1) {
        const float od = __shfl_xor_sync(FULL_MASK, d, o);
        const uint32_t oi = __shfl_xor_sync(FULL_MASK, idx, o);
        if (od < d || (od == d && oi < idx)) { d = od; idx = oi; }
    }
}

// testFacesDirectionPolyhedronVsPolyhedron (SATAlgorithm.cpp:1113-1142), faces spread over lanes
template <class PA, class PB>
RD float warp_sat_faces(const PA& pa, const PB& pb, const xform& a2b, uint32_t& minFace, int lane) {
    const uint32_t nf = pa.nfaces();
    float best = DECIMAL_LARGEST;
    uint32_t bestF = 0xffffffffu;
    for (uint32_t base = 0; base < nf; base += 32) {
        const uint32_t f = base + lane;
        const bool valid = f < nf;
        const float d = valid ? sat_single_face(pa, pb, a2b, f) : DECIMAL_LARGEST;
        const unsigned sep = __ballot_sync(FULL_MASK, valid && d <= 0.0f);
        if (sep) {
            const int l = __ffs(sep) - 1;
            minFace = base + l;
            return __shfl_sync(FULL_MASK, d, l);
        }
        if (valid && d < best) { best = d; bestF = f; }
    }
    warp_argmin(best, bestF);
    minFace = bestF;
    return best;
}

// Support point of a convex mesh with the vertices spread over lanes
// (ConvexMeshShape::getLocalSupportPointWithoutMargin, ConvexMeshShape.cpp:80-102):
// the first vertex with the largest dot product; a dot product only counts
// when it beats DECIMAL_SMALLEST, exactly like the reference's running maximum.
RD v3 warp_mesh_support(const MeshPoly& m, v3 d, int lane) {
    float best = DECIMAL_SMALLEST;
    uint32_t bi = 0xffffffffu;
    const uint32_t nv = m.h->nv, o = m.h->off_verts;
    for (uint32_t i = lane; i < nv; i += 32) {
        const float dp = vdot(d, V(m.f(o + 3 * i), m.f(o + 3 * i + 1), m.f(o + 3 * i + 2)));
        if (dp > best) { best = dp; bi = i; }
    }
    for (int s = 16; s; s >>= 1) {
        const float ob = __shfl_xor_sync(FULL_MASK, best, s);
        const uint32_t oi = __shfl_xor_sync(FULL_MASK, bi, s);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    return m.vertex(bi == 0xffffffffu ? 0u : bi);
}

// testFacesDirectionPolyhedronVsPolyhedron for the faces of a box against a
// convex mesh: faces in order (first separating face, strict minimum), the
// mesh support search spread over the lanes.
RD float warp_sat_faces(const BoxPoly& pa, const MeshPoly& pb, const xform& a2b, uint32_t& minFace, int lane) {
    // the six support searches run side by side (independent accumulators)
    v3 dir[6];
    float best[6];
    uint32_t bi[6];
#pragma unroll
    for (uint32_t f = 0; f < 6; f++) {
        dir[f] = vneg(qrot(a2b.q, pa.normal(f)));
        best[f] = DECIMAL_SMALLEST;
        bi[f] = 0xffffffffu;
    }
    const uint32_t nv = pb.h->nv, o = pb.h->off_verts;
    for (uint32_t i = lane; i < nv; i += 32) {
        const v3 v = V(pb.f(o + 3 * i), pb.f(o + 3 * i + 1), pb.f(o + 3 * i + 2));
#pragma unroll
        for (uint32_t f = 0; f < 6; f++) {
            const float dp = vdot(dir[f], v);
            if (dp > best[f]) { best[f] = dp; bi[f] = i; }
        }
    }
#pragma unroll
    for (int sft = 16; sft; sft >>= 1) {
#pragma unroll
        for (uint32_t f = 0; f < 6; f++) {
            const float ob = __shfl_xor_sync(FULL_MASK, best[f], sft);
            const uint32_t oi = __shfl_xor_sync(FULL_MASK, bi[f], sft);
            if (ob > best[f] || (ob == best[f] && oi < bi[f])) { best[f] = ob; bi[f] = oi; }
        }
    }
    float minDepth = DECIMAL_LARGEST;
    for (uint32_t f = 0; f < 6; f++) {
        const v3 fn2 = qrot(a2b.q, pa.normal(f));
        const v3 sp = pb.vertex(bi[f] == 0xffffffffu ? 0u : bi[f]);
        const v3 fv = xapply(a2b, pa.vertex(pa.face_vertex(f, 0)));
        const float d = vdot(vsub(fv, sp), fn2);
        if (d <= 0.0f) { minFace = f; return d; }
        if (d < minDepth) { minDepth = d; minFace = f; }
    }
    return minDepth;
}

template <class P2>
RD void edge2_data(const P2& p2, uint32_t j, hedge& e2, v3& e2A, v3& dir2) {
    e2 = p2.edge(j);
    e2A = p2.vertex(e2.vertex);
    dir2 = vsub(p2.vertex(p2.edge(e2.next).vertex), e2A);
}

// findMostAntiParallelFace with the faces spread over lanes: minimum dot
// product, first face on ties (the reference's strict '<' keeps the first).
template <class P>
RD uint32_t warp_most_antiparallel_face(const P& p, v3 dir, int lane) {
    float best = DECIMAL_LARGEST;
    uint32_t bestF = 0xffffffffu;
    const uint32_t nf = p.nfaces();
    for (uint32_t f = lane; f < nf; f += 32) {
        const float d = vdot(p.normal(f), dir);
        if (d < best) { best = d; bestF = f; }
    }
    warp_argmin(best, bestF);
    return bestF == 0xffffffffu ? 0u : bestF;
}

RD uint32_t warp_exclusive_scan(uint32_t v, int lane, uint32_t& total) {
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL_MASK, x, o);
        if (lane >= o) x += y;
    }
    total = __shfl_sync(FULL_MASK, x, 31);
    return x - v;
}

// computePolyhedronVsPolyhedronFaceContactPoints (SATAlgorithm.cpp:893-1036)
// on a whole warp.  Each Sutherland-Hodgman pass (clipPolygonWithPlane,
// mathematics_functions.h:332-393) gives lane l the polygon edge that ends at
// vertex l; its 0, 1 or 2 output points go to position (exclusive prefix sum
// of the counts), which is exactly the sequential output order.  Vertex dot
// products are the same expressions as in the sequential pass.  Contacts are
// appended in clipped-vertex order.  All lanes return the same value.
// Functions a pair runs at most once or twice (the clipping of the contact
// face) may be kept out of line to shrink the instruction footprint of the
// warp-per-pair kernel (RP3DG_NP_COLD_NOINLINE, a build option).
#ifdef RP3DG_NP_COLD_NOINLINE
#define RD_COLD __device__ __noinline__
#else
#define RD_COLD RD
#endif
template <class PR, class PI>
RD_COLD bool warp_face_contacts(bool ref1, const PR& refP, const PI& incP, const xform& r2i, const xform& i2r,
                           uint32_t minFace, Item& it, int lane, v3* poly) {
    const v3 axisR = refP.normal(minFace);
    const v3 axisI = qrot(r2i.q, axisR);
    const v3 nw = ref1 ? qrot(it.t1.q, axisR) : vneg(qrot(it.t2.q, axisR));
    const uint32_t incFace = warp_most_antiparallel_face(incP, axisI, lane);
    uint32_t n = incP.face_count(incFace);
    if (n > CLIP_MAX) n = CLIP_MAX;
    NP_EV(it, EV_CLIP_SETUP, 1);
    NP_EV(it, EV_ANTIPARALLEL, incP.nfaces());
    NP_EV(it, EV_INC_VERTEX, n);
    v3 P = V(0.0f, 0.0f, 0.0f);
    if (uint32_t(lane) < n) P = xapply(i2r, incP.vertex(incP.face_vertex(incFace, lane)));
    const uint32_t firstEdge = refP.face_edge(minFace);
    hedge cur = refP.edge(firstEdge);
    v3 ev1 = refP.vertex(cur.vertex);
    uint32_t curIdx, guard = 0;
    do {
        const hedge nxt = refP.edge(cur.next);
        const v3 ev2 = refP.vertex(nxt.vertex);
        const v3 pn = vcross(axisR, vsub(ev2, ev1));
        const float pnpp = vdot(pn, ev1);
        const bool active = uint32_t(lane) < n;
        NP_EV(it, EV_CLIP_PLANE, 1);
        NP_EV(it, EV_CLIP_VERTEX, n);
        const float ven = active ? vdot(vsub(P, ev1), pn) : 0.0f;
        const int src = lane == 0 ? int(n) - 1 : lane - 1;
        const v3 S = V(__shfl_sync(FULL_MASK, P.x, src), __shfl_sync(FULL_MASK, P.y, src), __shfl_sync(FULL_MASK, P.z, src));
        const float vsn = __shfl_sync(FULL_MASK, ven, src);
        v3 o0 = V(0.0f, 0.0f, 0.0f), o1 = V(0.0f, 0.0f, 0.0f);
        uint32_t cnt = 0;
        if (active) {
            if (ven >= 0.0f) {
                if (vsn < 0.0f) {
                    const float t = plane_segment_intersection(S, P, pnpp, pn);
                    o0 = (t >= 0.0f && t <= 1.0f) ? vadd(S, vmul(vsub(P, S), t)) : P;
                    o1 = P;
                    cnt = 2;
                } else {
                    o0 = P;
                    cnt = 1;
                }
            } else if (vsn >= 0.0f) {
                const float t = plane_segment_intersection(S, P, -pnpp, vneg(pn));
                o0 = (t >= 0.0f && t <= 1.0f) ? vadd(S, vmul(vsub(P, S), t)) : S;
                cnt = 1;
            }
        }
        NP_EV(it, EV_CLIP_INTERSECT, __popc(__ballot_sync(FULL_MASK, active && (ven >= 0.0f) != (vsn >= 0.0f))));
        uint32_t total;
        const uint32_t pos = warp_exclusive_scan(cnt, lane, total);
        __syncwarp();
        if (cnt >= 1 && pos < CLIP_MAX) poly[pos] = o0;
        if (cnt == 2 && pos + 1 < CLIP_MAX) poly[pos + 1] = o1;
        __syncwarp();
        n = total < CLIP_MAX ? total : CLIP_MAX;
        if (uint32_t(lane) < n) P = poly[lane];
        __syncwarp();
        curIdx = cur.next;
        cur = nxt;
        ev1 = ev2;
    } while (curIdx != firstEdge && n > 0 && ++guard < MAX_FACE_VERTICES);
    const v3 refV = refP.vertex(refP.edge(firstEdge).vertex);
    const bool active = uint32_t(lane) < n;
    const float depth = active ? vdot(vsub(refV, P), axisR) : 0.0f;
    const bool hit = active && depth > 0.0f;
    const unsigned mask = __ballot_sync(FULL_MASK, hit);
    NP_EV(it, EV_CLIP_DEPTH, n);
    if (it.report) NP_EV(it, EV_CONTACT, __popc(mask));
    if (mask && it.report) {
        const uint32_t slot = it.out.count + __popc(mask & ((1u << lane) - 1u));
        if (hit && slot < MAX_CONTACTS) {
            const v3 pInc = xapply(r2i, P);
            const v3 pRef = project_onto_plane(P, axisR, refV);
            ContactSink s = it.out;
            s.count = slot;
            s.add(nw, depth, ref1 ? pRef : pInc, ref1 ? pInc : pRef);
        }
        const uint32_t c = it.out.count + __popc(mask);
        it.out.count = c < MAX_CONTACTS ? c : MAX_CONTACTS;
    }
    return mask != 0;
}

template <class P1, class P2>
RD bool warp_poly_face_contacts(bool ref1, const P1& p1, const P2& p2, const xform& p1to2, const xform& p2to1,
                                uint32_t minFace, Item& it, int lane, v3* poly) {
    if (ref1) return warp_face_contacts(true, p1, p2, p1to2, p2to1, minFace, it, lane, poly);
    return warp_face_contacts(false, p2, p1, p2to1, p1to2, minFace, it, lane, poly);
}

// Walks the edge pairs (i, j) of the reference's double loop in visiting
// order, a round at a time; lane `offset` of a round holds pair base + offset.
// Generic polyhedron 2: 32 consecutive pairs per round.
template <class P2>
struct EdgePairWalker {
    const P2& p2;
    uint32_t n2h, ih, jh, qstep, rstep, offset, per_round;
    bool active;
    RD EdgePairWalker(const P2& p, uint32_t n2, int lane) : p2(p), n2h(n2) {
        ih = uint32_t(lane) / n2h;
        jh = uint32_t(lane) - ih * n2h;
        qstep = 32u / n2h;
        rstep = 32u - qstep * n2h;
        offset = uint32_t(lane);
        per_round = 32;
        active = true;
    }
    RD bool test(const Edge1Stage* stage) const {
        const Edge1Stage& s = stage[ih];
        Edge1Gauss g;
        g.a = V(s.a[0], s.a[1], s.a[2]);
        g.b = V(s.b[0], s.b[1], s.b[2]);
        g.bxa = V(s.bxa[0], s.bxa[1], s.bxa[2]);
        return edges_minkowski(g, p2, p2.edge(2 * jh), 2 * jh);
    }
    RD void advance() {
        jh += rstep; ih += qstep;
        if (jh >= n2h) { jh -= n2h; ih++; }
    }
    static constexpr int UNROLL = 1;
    RD bool test_ahead(const Edge1Stage* stage, int) const { return test(stage); }
    RD void advance_by(int u) { for (int k = 0; k < u; k++) advance(); }
};
// Box polyhedron 2: its 12 even half-edges are fixed per lane (lanes 0..23 =
// two rows i of the loop), so each lane keeps its box edge's Gauss-map data in
// registers and reads only the three components of the staged edge it needs.
template <>
struct EdgePairWalker<BoxPoly> {
    uint32_t ih, offset, per_round;
    bool active;
    uint32_t k, m, n;
    bool negC, negD2;
    float D;
    RD EdgePairWalker(const BoxPoly& p2, uint32_t, int lane) {
        active = lane < 24;
        const uint32_t jh = uint32_t(lane) % 12u, half = uint32_t(lane) / 12u;
        ih = half;
        offset = uint32_t(lane);
        per_round = 24;
        const uint8_t* gi = p2.t->gauss[2 * jh];
        k = gi[0] & 3u; m = gi[1] & 3u; n = gi[2] & 3u;
        negC = (gi[1] & 4u) != 0;
        negD2 = (gi[2] & 4u) != 0;
        const float hk = axis_component(p2.he, k);
        D = (gi[0] & 4u) ? -(hk + hk) : (hk + hk);
    }
    RD bool test(const Edge1Stage* stage) const { return test_ahead(stage, 0); }
    RD bool test_ahead(const Edge1Stage* stage, int u) const {
        const Edge1Stage& s = stage[ih + 2 * u];
        const float bm = s.bxa[m], bn = s.bxa[n];
        const float cba = negC ? -bm : bm;
        const float dba = negD2 ? -bn : bn;
        const float adc = s.a[k] * D;
        const float bdc = s.b[k] * D;
        return cba * dba < 0.0f && adc * bdc < 0.0f && cba * bdc > 0.0f;
    }
    RD void advance() { ih += 2; }
    static constexpr int UNROLL = 4;
    RD void advance_by(int u) { ih += 2 * u; }
};

// testCollisionConvexPolyhedronVsConvexPolyhedron (SATAlgorithm.cpp:485-889), one warp per pair.
// Every lane holds the same pair state; contacts and outputs are produced by lane 0.
template <class P1, class P2>
RD void warp_sat_poly_poly(Item& it, const P1& p1, const P2& p2, bool clipPrev, int lane, WarpScratch& ws) {
    NP_EV(it, EV_POLY_SETUP, 1);
    Edge1Stage* stage = ws.stage;
    PhaseTimer timer(lane);
    const xform p1to2 = xmul(xinv(it.t2), it.t1);
    const xform p2to1 = xinv(p1to2);
    LastFrame& lf = it.lf;

    const bool cacheInRange = lf.has(RP3DG_LF_SAT_FACE_POLY1)   ? lf.sat_face < p1.nfaces()
                              : lf.has(RP3DG_LF_SAT_FACE_POLY2) ? lf.sat_face < p2.nfaces()
                                                                : (lf.sat_e1 < p1.nhe() && lf.sat_e2 < p2.nhe());
    if (cacheInRange && lf.has(RP3DG_LF_IS_VALID) && lf.has(RP3DG_LF_WAS_USING_SAT)) {
        const bool wasColliding = lf.has(RP3DG_LF_WAS_COLLIDING);
        if (lf.has(RP3DG_LF_SAT_FACE_POLY1) || lf.has(RP3DG_LF_SAT_FACE_POLY2)) {
            const bool face1 = lf.has(RP3DG_LF_SAT_FACE_POLY1);
            const float d = face1 ? sat_single_face(p1, p2, p1to2, lf.sat_face) : sat_single_face(p2, p1, p2to1, lf.sat_face);
            if (face1) ev_face_tests(it, p2, 1);
            else ev_face_tests(it, p1, 1);
            if (!wasColliding && d <= 0.0f) return;
            if (wasColliding && clipPrev && d > 0.0f) {
                const bool found = warp_poly_face_contacts(face1, p1, p2, p1to2, p2to1, lf.sat_face, it, lane, ws.poly);
                if (found) {
                    lf.set(RP3DG_LF_SAT_FACE_POLY1, face1);
                    lf.set(RP3DG_LF_SAT_FACE_POLY2, !face1);
                    it.colliding = true;
                    return;
                }
            }
        } else {
            const hedge e1 = p1.edge(lf.sat_e1);
            const hedge e2 = p2.edge(lf.sat_e2);
            const v3 e1A = xapply(p1to2, p1.vertex(e1.vertex));
            const v3 e1B = xapply(p1to2, p1.vertex(p1.edge(e1.next).vertex));
            const v3 d1 = vsub(e1B, e1A);
            const v3 e2A = p2.vertex(e2.vertex);
            const v3 e2B = p2.vertex(p2.edge(e2.next).vertex);
            const v3 d2 = vsub(e2B, e2A);
            NP_EV(it, EV_EDGE1, 1);
            NP_EV(it, EV_GAUSS, 1);
            if (edges_minkowski(edge1_gauss(p1, e1, p1to2), p2, e2, lf.sat_e2)) {
                NP_EV(it, EV_EDGE_DIST, 1);
                v3 axis;
                const v3 c1 = xapply(p1to2, p1.centroid());
                const float d = sat_edge_distance(e1A, e2A, c1, d1, d2, axis);
                if (!wasColliding && d <= 0.0f) return;
                if (wasColliding && clipPrev && d > 0.0f && d < DECIMAL_LARGEST) {
                    v3 cp1, cp2;
                    closest_points_segments(e1A, e1B, e2A, e2B, cp1, cp2);
                    const float l1 = vlen2(d1), l2 = vlen2(d2);
                    const float t1 = vdot(vsub(cp1, e2A), d2) / l2;
                    const float t2 = vdot(vsub(cp2, e1A), d1) / l1;
                    NP_EV(it, EV_EDGE_CONTACT, 1);
                    if (t1 >= 0.0f && t1 <= 1.0f && t2 >= 0.0f && t2 <= 1.0f) {
                        if (it.report) it.out.add(qrot(it.t2.q, axis), d, xapply(p2to1, cp1), cp2, lane == 0);
                        it.colliding = true;
                        return;
                    }
                }
            }
        }
    }

    if (it.proposal < 15) {
        it.proposal_tested = true;
        if (confirm_proposal(it.proposal, p1, p2, p1to2, p2to1, lf, IsBox<P1>::value, IsBox<P2>::value, box_tables_of(p1, p2))) {
            it.proposal_confirmed = true;
            return;
        }
    }
    timer.mark(0);
    uint32_t f1 = 0, f2 = 0;
    const float d1 = warp_sat_faces(p1, p2, p1to2, f1, lane);
    ev_face_tests(it, p2, d1 <= 0.0f ? f1 + 1 : p1.nfaces());
    timer.mark(1);
    if (d1 <= 0.0f) {
        lf.set(RP3DG_LF_SAT_FACE_POLY1, true); lf.set(RP3DG_LF_SAT_FACE_POLY2, false); lf.sat_face = f1;
        return;
    }
    const float d2 = warp_sat_faces(p2, p1, p2to1, f2, lane);
    ev_face_tests(it, p1, d2 <= 0.0f ? f2 + 1 : p2.nfaces());
    timer.mark(2);
    if (d2 <= 0.0f) {
        lf.set(RP3DG_LF_SAT_FACE_POLY1, false); lf.set(RP3DG_LF_SAT_FACE_POLY2, true); lf.sat_face = f2;
        return;
    }
    const float faceMin = smin(d1, d2);
    uint32_t minFace;
    bool isFace1;
    if (d1 < d2 * SAT_REL_TOL + SAT_ABS_TOL) { minFace = f1; isFace1 = true; }
    else { minFace = f2; isFace1 = false; }

    // stage the even half-edges of polyhedron 1 (in polyhedron-2 space)
    const uint32_t n1h = (p1.nhe() + 1) / 2, n2h = (p2.nhe() + 1) / 2;
    const v3 c1 = xapply(p1to2, p1.centroid());
    for (uint32_t ih = lane; ih < n1h; ih += 32) {
        const hedge e1 = p1.edge(2 * ih);
        const v3 e1A = xapply(p1to2, p1.vertex(e1.vertex));
        const v3 e1B = xapply(p1to2, p1.vertex(p1.edge(e1.next).vertex));
        const v3 dir1 = vsub(e1B, e1A);
        const Edge1Gauss g = edge1_gauss(p1, e1, p1to2);
        Edge1Stage& s = stage[ih];
        s.e1A[0] = e1A.x; s.e1A[1] = e1A.y; s.e1A[2] = e1A.z;
        s.dir1[0] = dir1.x; s.dir1[1] = dir1.y; s.dir1[2] = dir1.z;
        s.a[0] = g.a.x; s.a[1] = g.a.y; s.a[2] = g.a.z;
        s.b[0] = g.b.x; s.b[1] = g.b.y; s.b[2] = g.b.z;
        s.bxa[0] = g.bxa.x; s.bxa[1] = g.bxa.y; s.bxa[2] = g.bxa.z;
    }
    __syncwarp();
    timer.mark(3);
    const uint32_t total = n1h * n2h;
    float best = DECIMAL_LARGEST;
    uint32_t bestIdx = 0xffffffffu;
    // Pass 1 walks the edge pairs in visiting order and appends the ones that
    // pass the Gauss-map test to ws.cand; pass 2 (run whenever the list could
    // overflow, and at the end) computes their distances 32 at a time.  The
    // list keeps visiting order, so the first separating pair and the
    // first arg-min are those of the sequential loop.
    uint32_t ncand = 0;
    bool separated = false;
    NP_EV_ONLY(uint32_t cand_before = 0;)
    EdgePairWalker<P2> walk(p2, n2h, lane);
    for (uint32_t base = 0; base < total || ncand > 0;) {
        if (EdgePairWalker<P2>::UNROLL > 1 && base < total && ncand + 32 * EdgePairWalker<P2>::UNROLL <= WARP_CAND_CAP) {
            // several rounds at once: independent loads and tests, then the
            // ballots in round order (keeps the visiting order)
            constexpr int U = EdgePairWalker<P2>::UNROLL;
            bool pass[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t idx = base + u * walk.per_round + walk.offset;
                pass[u] = walk.active && idx < total && walk.test_ahead(stage, u);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t idx = base + u * walk.per_round + walk.offset;
                const unsigned m = __ballot_sync(FULL_MASK, pass[u]);
                if (pass[u]) ws.cand[ncand + __popc(m & ((1u << lane) - 1u))] = uint16_t(idx);
                ncand += __popc(m);
            }
            base += U * walk.per_round;
            walk.advance_by(U);
            continue;
        }
        if (base < total && ncand + 32 <= WARP_CAND_CAP) {
            const uint32_t idx = base + walk.offset;
            const bool pass = walk.active && idx < total && walk.test(stage);
            const unsigned m = __ballot_sync(FULL_MASK, pass);
            if (pass) ws.cand[ncand + __popc(m & ((1u << lane) - 1u))] = uint16_t(idx);
            ncand += __popc(m);
            base += walk.per_round;
            walk.advance();
            continue;
        }
        __syncwarp();
        for (uint32_t c0 = 0; c0 < ncand && !separated; c0 += 32) {
            const uint32_t c = c0 + lane;
            float d = DECIMAL_LARGEST;
            uint32_t idx = 0xffffffffu;
            if (c < ncand) {
                idx = ws.cand[c];
                const uint32_t ci = idx / n2h, cj = idx - ci * n2h;
                const Edge1Stage& s = stage[ci];
                hedge e2;
                v3 e2A, dir2, axis;
                edge2_data(p2, 2 * cj, e2, e2A, dir2);
                d = sat_edge_distance(V(s.e1A[0], s.e1A[1], s.e1A[2]), e2A, c1, V(s.dir1[0], s.dir1[1], s.dir1[2]),
                                      dir2, axis);
            }
            const unsigned sep = __ballot_sync(FULL_MASK, c < ncand && d <= 0.0f);
            if (sep) {
                const uint32_t first = __shfl_sync(FULL_MASK, idx, __ffs(sep) - 1);
                const uint32_t fi = first / n2h;
                // the reference's loop stops at this pair
                NP_EV(it, EV_EDGE1, fi + 1);
                NP_EV(it, EV_GAUSS, first + 1);
                NP_EV(it, EV_EDGE_DIST, cand_before + c0 + uint32_t(__ffs(sep)));
                lf.set(RP3DG_LF_SAT_FACE_POLY1, false); lf.set(RP3DG_LF_SAT_FACE_POLY2, false);
                lf.sat_e1 = 2 * fi;
                lf.sat_e2 = 2 * (first - fi * n2h);
                separated = true;
            } else if (c < ncand && d < best) {
                best = d; bestIdx = idx;
            }
        }
        __syncwarp();
        if (separated) return;
        NP_EV_ONLY(cand_before += ncand;)
        ncand = 0;
    }
    NP_EV(it, EV_EDGE1, n1h);
    NP_EV(it, EV_GAUSS, total);
    NP_EV(it, EV_EDGE_DIST, cand_before);
    warp_argmin(best, bestIdx);
    __syncwarp();
    timer.mark(4);
    const bool edgeWins = bestIdx != 0xffffffffu && best * SAT_REL_TOL + SAT_ABS_TOL < faceMin;

    if (!edgeWins) {
        const bool found = warp_poly_face_contacts(isFace1, p1, p2, p1to2, p2to1, minFace, it, lane, ws.poly);
        lf.set(RP3DG_LF_SAT_FACE_POLY1, isFace1); lf.set(RP3DG_LF_SAT_FACE_POLY2, !isFace1); lf.sat_face = minFace;
        if (!found) return;
    } else {
        const uint32_t ih = bestIdx / n2h, jh = bestIdx - ih * n2h;
        if (it.report) {
            NP_EV(it, EV_EDGE_CONTACT, 1);
            const hedge e1 = p1.edge(2 * ih);
            const v3 e1A = xapply(p1to2, p1.vertex(e1.vertex));
            const v3 e1B = xapply(p1to2, p1.vertex(p1.edge(e1.next).vertex));
            hedge e2;
            v3 e2A, dir2;
            edge2_data(p2, 2 * jh, e2, e2A, dir2);
            const v3 e2B = p2.vertex(p2.edge(e2.next).vertex);
            v3 axis;
            sat_edge_distance(e1A, e2A, c1, vsub(e1B, e1A), dir2, axis);
            v3 cp1, cp2;
            closest_points_segments(e1A, e1B, e2A, e2B, cp1, cp2);
            it.out.add(qrot(it.t2.q, axis), best, xapply(p2to1, cp1), cp2, lane == 0);
        }
        lf.set(RP3DG_LF_SAT_FACE_POLY1, false); lf.set(RP3DG_LF_SAT_FACE_POLY2, false);
        lf.sat_e1 = 2 * ih; lf.sat_e2 = 2 * jh;
    }
    timer.mark(5);
    it.colliding = true;
}

}  // namespace rp3dg
