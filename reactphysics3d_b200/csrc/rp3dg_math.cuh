// Single-precision vector, quaternion and transform arithmetic with the exact
// expression trees of ReactPhysics3D v0.10.2's mathematics headers, so that
// device results (compiled with --fmad=false and IEEE div/sqrt) are
// bit-identical to the reference's x86-64 float build.
//
// Paths below are inside the reference project.
#pragma once
#include <cfloat>
#include <cstdint>

#define RD __device__ __forceinline__

namespace rp3dg {

constexpr float MACHINE_EPSILON = FLT_EPSILON;   // configuration.h:120
constexpr float DECIMAL_LARGEST = FLT_MAX;       // configuration.h:117
constexpr float DECIMAL_SMALLEST = -FLT_MAX;     // configuration.h:114

struct v3 { float x, y, z; };
struct quat { float x, y, z, w; };
struct xform { v3 p; quat q; };

RD v3 V(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
RD v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
RD v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
RD v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
// operator*(Vector3, decimal): Vector3(number * v.x, ...)  (Vector3.h:322-324)
RD v3 vmul(v3 a, float s) { return V(s * a.x, s * a.y, s * a.z); }
RD v3 vdivs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
RD v3 vcmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
RD float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RD v3 vcross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
RD float vlen2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
RD float vlen(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
// Vector3::getUnit (Vector3.cpp:33-43): multiply by a rounded reciprocal
RD v3 vunit(v3 a) {
    const float l = vlen(a);
    if (l < MACHINE_EPSILON) return a;
    const float inv = 1.0f / l;
    return V(a.x * inv, a.y * inv, a.z * inv);
}
// Vector3::normalize (Vector3.h:219-227): three divisions
RD v3 vnormalize(v3 a) {
    const float l = vlen(a);
    if (l < MACHINE_EPSILON) return a;
    return V(a.x / l, a.y / l, a.z / l);
}
// std::min / std::max semantics (not fminf/fmaxf: signed zeros and NaN differ)
RD float smin(float a, float b) { return (b < a) ? b : a; }
RD float smax(float a, float b) { return (a < b) ? b : a; }
RD float sclamp(float v, float lo, float hi) { return smin(smax(v, lo), hi); }

RD quat Q(float x, float y, float z, float w) { quat r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }
RD quat qinv(quat q) { return Q(-q.x, -q.y, -q.z, q.w); }  // Quaternion.h:283-287
// Quaternion * Quaternion (Quaternion.h:346-359)
RD quat qmul(quat a, quat b) {
    return Q(a.w * b.x + b.w * a.x + a.y * b.z - a.z * b.y,
             a.w * b.y + b.w * a.y + a.z * b.x - a.x * b.z,
             a.w * b.z + b.w * a.z + a.x * b.y - a.y * b.x,
             a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
// Quaternion * Vector3 (Quaternion.h:363-379)
RD v3 qrot(quat q, v3 p) {
    const float prodX = q.w * p.x + q.y * p.z - q.z * p.y;
    const float prodY = q.w * p.y + q.z * p.x - q.x * p.z;
    const float prodZ = q.w * p.z + q.x * p.y - q.y * p.x;
    const float prodW = -q.x * p.x - q.y * p.y - q.z * p.z;
    return V(q.w * prodX - prodY * q.z + prodZ * q.y - prodW * q.x,
             q.w * prodY - prodZ * q.x + prodX * q.z - prodW * q.y,
             q.w * prodZ - prodX * q.y + prodY * q.x - prodW * q.z);
}
RD xform X(v3 p, quat q) { xform t; t.p = p; t.q = q; return t; }
// Transform::getInverse (Transform.h:162-165)
RD xform xinv(xform t) { const quat iq = qinv(t.q); return X(qrot(iq, vneg(t.p)), iq); }
// Transform * Vector3 (Transform.h:193-195)
RD v3 xapply(xform t, v3 v) { return vadd(qrot(t.q, v), t.p); }
// Transform * Transform (Transform.h:198-225)
RD xform xmul(xform a, xform b) {
    const quat o = a.q;
    const v3 p = b.p;
    const float prodX = o.w * p.x + o.y * p.z - o.z * p.y;
    const float prodY = o.w * p.y + o.z * p.x - o.x * p.z;
    const float prodZ = o.w * p.z + o.x * p.y - o.y * p.x;
    const float prodW = -o.x * p.x - o.y * p.y - o.z * p.z;
    const v3 np = V(a.p.x + o.w * prodX - prodY * o.z + prodZ * o.y - prodW * o.x,
                    a.p.y + o.w * prodY - prodZ * o.x + prodX * o.z - prodW * o.y,
                    a.p.z + o.w * prodZ - prodX * o.y + prodY * o.x - prodW * o.z);
    const quat q2 = b.q;
    const quat nq = Q(o.w * q2.x + q2.w * o.x + o.y * q2.z - o.z * q2.y,
                      o.w * q2.y + q2.w * o.y + o.z * q2.x - o.x * q2.z,
                      o.w * q2.z + q2.w * o.z + o.x * q2.y - o.y * q2.x,
                      o.w * q2.w - o.x * q2.x - o.y * q2.y - o.z * q2.z);
    return X(np, nq);
}

// areParallelVectors / areOrthogonalVectors (mathematics_functions.h:76-84)
RD bool are_parallel(v3 a, v3 b) { return vlen2(vcross(a, b)) < 0.00001f; }
RD bool are_orthogonal(v3 a, v3 b) { return fabsf(vdot(a, b)) < 0.001f; }

// computeClosestPointOnSegment (mathematics_functions.h:96-118)
RD v3 closest_point_on_segment(v3 a, v3 b, v3 c) {
    const v3 ab = vsub(b, a);
    const float abl2 = vlen2(ab);
    if (abl2 < MACHINE_EPSILON) return a;
    float t = vdot(vsub(c, a), ab) / abl2;
    if (t < 0.0f) t = 0.0f;
    if (t > 1.0f) t = 1.0f;
    return vadd(a, vmul(ab, t));
}

// computeClosestPointBetweenTwoSegments (mathematics_functions.h:123-190)
RD void closest_points_segments(v3 s1a, v3 s1b, v3 s2a, v3 s2b, v3& c1, v3& c2) {
    const v3 d1 = vsub(s1b, s1a);
    const v3 d2 = vsub(s2b, s2a);
    const v3 r = vsub(s1a, s2a);
    const float a = vlen2(d1);
    const float e = vlen2(d2);
    const float f = vdot(d2, r);
    float s, t;
    if (a <= MACHINE_EPSILON && e <= MACHINE_EPSILON) { c1 = s1a; c2 = s2a; return; }
    if (a <= MACHINE_EPSILON) {
        s = 0.0f;
        t = sclamp(f / e, 0.0f, 1.0f);
    } else {
        const float c = vdot(d1, r);
        if (e <= MACHINE_EPSILON) {
            t = 0.0f;
            s = sclamp(-c / a, 0.0f, 1.0f);
        } else {
            const float b = vdot(d1, d2);
            const float denom = a * e - b * b;
            if (denom != 0.0f) s = sclamp((b * f - c * e) / denom, 0.0f, 1.0f);
            else s = 0.0f;
            t = (b * s + f) / e;
            if (t < 0.0f) { t = 0.0f; s = sclamp(-c / a, 0.0f, 1.0f); }
            else if (t > 1.0f) { t = 1.0f; s = sclamp((b - c) / a, 0.0f, 1.0f); }
        }
    }
    c1 = vadd(s1a, vmul(d1, s));
    c2 = vadd(s2a, vmul(d2, t));
}

// computePlaneSegmentIntersection (mathematics_functions.h:224-237)
RD float plane_segment_intersection(v3 a, v3 b, float d, v3 n) {
    float t = -1.0f;
    const float nab = vdot(n, vsub(b, a));
    if (fabsf(nab) > 0.0001f) t = (d - vdot(n, a)) / nab;
    return t;
}

// computePointToLineDistance (mathematics_functions.h:240-249)
RD float point_to_line_distance(v3 a, v3 b, v3 p) {
    const float dab = vlen(vsub(b, a));
    if (dab < MACHINE_EPSILON) return vlen(vsub(p, a));
    return vlen(vcross(vsub(p, a), vsub(p, b))) / dab;
}

// projectPointOntoPlane (mathematics_functions.h:396-398)
RD v3 project_onto_plane(v3 p, v3 n, v3 pp) { return vsub(p, vmul(n, vdot(n, vsub(p, pp)))); }

}  // namespace rp3dg
