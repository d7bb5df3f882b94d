// Joints of the dynamics stage: ball-and-socket (SolveBallAndSocketJointSystem,
// reference src/systems/SolveBallAndSocketJointSystem.cpp), hinge
// (src/systems/SolveHingeJointSystem.cpp), fixed
// (src/systems/SolveFixedJointSystem.cpp) and slider
// (src/systems/SolveSliderJointSystem.cpp): the per-step
// initialisation (initBeforeSolve), warm start, velocity solve and the
// non-linear Gauss-Seidel position correction, one joint at a time, with the
// reference's float expression trees (Matrix3x3 / Matrix2x2 / Quaternion /
// Vector3 operators of include/reactphysics3d/mathematics).  Only the
// NON_LINEAR_GAUSS_SEIDEL position correction (the reference's default) is
// built.  The cone half angle (std::acos) and the hinge angle (std::atan2) go
// through CUDA's acosf / atan2f, which may differ from the host C library in
// the last bit; they only matter when a cone limit, a hinge limit or a motor
// is enabled.
#pragma once
#include "dynamics_launch.h"
#include "rp3dg_math.cuh"

namespace rp3dg {

// --- 3x3 / 2x2 matrix helpers, row-major, reference operator order --------
struct M3 {
    float m[9];
};
RD M3 m3_zero() { M3 r; for (int i = 0; i < 9; i++) r.m[i] = 0.0f; return r; }
// Matrix3x3::computeSkewSymmetricMatrixForCrossProduct (Matrix3x3.h:251-253)
RD M3 m3_skew(v3 v) {
    M3 r;
    r.m[0] = 0.0f; r.m[1] = -v.z; r.m[2] = v.y;
    r.m[3] = v.z; r.m[4] = 0.0f; r.m[5] = -v.x;
    r.m[6] = -v.y; r.m[7] = v.x; r.m[8] = 0.0f;
    return r;
}
RD M3 m3_transpose(const M3& a) {
    M3 r;
    r.m[0] = a.m[0]; r.m[1] = a.m[3]; r.m[2] = a.m[6];
    r.m[3] = a.m[1]; r.m[4] = a.m[4]; r.m[5] = a.m[7];
    r.m[6] = a.m[2]; r.m[7] = a.m[5]; r.m[8] = a.m[8];
    return r;
}
// operator*(Matrix3x3, Matrix3x3) (Matrix3x3.h:302-318)
RD M3 m3_mul(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            r.m[3 * i + j] = a.m[3 * i + 0] * b.m[0 + j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return r;
}
RD M3 m3_add(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 9; i++) r.m[i] = a.m[i] + b.m[i];
    return r;
}
// Matrix3x3::getDeterminant (Matrix3x3.h:211-217)
RD float m3_det(const M3& a) {
    const float* m = a.m;
    return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[1] * (m[3] * m[8] - m[6] * m[5]) + m[2] * (m[3] * m[7] - m[6] * m[4]);
}
// Matrix3x3::getInverse(determinant) (Matrix3x3.cpp) then invDeterminant * tempMatrix
RD M3 m3_inverse(const M3& a, float det) {
    const float* m = a.m;
    const float inv = 1.0f / det;
    M3 t;
    t.m[0] = (m[4] * m[8] - m[7] * m[5]);
    t.m[1] = -(m[1] * m[8] - m[7] * m[2]);
    t.m[2] = (m[1] * m[5] - m[2] * m[4]);
    t.m[3] = -(m[3] * m[8] - m[6] * m[5]);
    t.m[4] = (m[0] * m[8] - m[6] * m[2]);
    t.m[5] = -(m[0] * m[5] - m[3] * m[2]);
    t.m[6] = (m[3] * m[7] - m[6] * m[4]);
    t.m[7] = -(m[0] * m[7] - m[6] * m[1]);
    t.m[8] = (m[0] * m[4] - m[1] * m[3]);
    for (int i = 0; i < 9; i++) t.m[i] = t.m[i] * inv;
    return t;
}
// operator*(Matrix3x3, Vector3) (Matrix3x3.h:324-331)
RD v3 m3_mulv(const M3& a, v3 v) {
    const float* m = a.m;
    return V(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
             m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
// K = diag(invMass) + (U1 * I1) * U1^T + (U2 * I2) * U2^T (left to right)
RD M3 joint_mass_matrix(float inv_mass, const M3& U1, const M3& I1, const M3& U2, const M3& I2) {
    M3 d = m3_zero();
    d.m[0] = inv_mass; d.m[4] = inv_mass; d.m[8] = inv_mass;
    const M3 a = m3_mul(m3_mul(U1, I1), m3_transpose(U1));
    const M3 b = m3_mul(m3_mul(U2, I2), m3_transpose(U2));
    return m3_add(m3_add(d, a), b);
}

RD v3 lin(float im, v3 lf, v3 imp) {  // inverseMass * lockFactor * impulse
    return V(im * lf.x * imp.x, im * lf.y * imp.y, im * lf.z * imp.z);
}
RD v3 v3add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
RD v3 sv(float s, v3 a) { return V(s * a.x, s * a.y, s * a.z); }
// q += Quaternion(0, w) * q * 0.5; q.normalize()  (Quaternion.h:238-249, 326-361)
RD quat q_add_rot(quat q, v3 w) {
    const quat d = qmul(Q(w.x, w.y, w.z, 0.0f), q);
    quat r = Q(q.x + 0.5f * d.x, q.y + 0.5f * d.y, q.z + 0.5f * d.z, q.w + 0.5f * d.w);
    const float l = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w);
    return Q(r.x / l, r.y / l, r.z / l, r.w / l);
}
RD quat qnormalize(quat r) {
    const float l = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w);
    return Q(r.x / l, r.y / l, r.z / l, r.w / l);
}

// --- joint records -------------------------------------------------------
constexpr float JOINT_PI = float(3.141592653589);
constexpr float JOINT_PI_TIMES_2 = float(6.28318530);

RD void st3(float4* q, const M3& a) {
    q[0] = make_float4(a.m[0], a.m[1], a.m[2], 0.0f);
    q[1] = make_float4(a.m[3], a.m[4], a.m[5], 0.0f);
    q[2] = make_float4(a.m[6], a.m[7], a.m[8], 0.0f);
}
RD M3 ld3(const float4* q) {
    M3 a;
    const float4 r0 = q[0], r1 = q[1], r2 = q[2];
    a.m[0] = r0.x; a.m[1] = r0.y; a.m[2] = r0.z;
    a.m[3] = r1.x; a.m[4] = r1.y; a.m[5] = r1.z;
    a.m[6] = r2.x; a.m[7] = r2.y; a.m[8] = r2.z;
    return a;
}
RD float4 F4v(v3 a, float w = 0.0f) { return make_float4(a.x, a.y, a.z, w); }
RD v3 L3v(float4 a) { return V(a.x, a.y, a.z); }

RD M3 iiw_of(const DynArgs& a, int32_t b) {
    return ld3(a.iiw + 3 * b);
}

// HingeJoint helpers (SolveHingeJointSystem.cpp:719-799)
RD float hinge_normalized(float angle) {
    angle = fmodf(angle, JOINT_PI_TIMES_2);
    if (angle < -JOINT_PI) return angle + JOINT_PI_TIMES_2;
    if (angle > JOINT_PI) return angle - JOINT_PI_TIMES_2;
    return angle;
}
RD float hinge_near_limits(float a, float lo, float hi) {
    if (hi <= lo) return a;
    if (a > hi) {
        const float du = fabsf(hinge_normalized(a - hi)), dl = fabsf(hinge_normalized(a - lo));
        return (du > dl) ? (a - JOINT_PI_TIMES_2) : a;
    }
    if (a < lo) {
        const float du = fabsf(hinge_normalized(hi - a)), dl = fabsf(hinge_normalized(lo - a));
        return (du > dl) ? a : (a + JOINT_PI_TIMES_2);
    }
    return a;
}
RD float hinge_angle(quat q1, quat q2, quat init_inv, v3 a1, float lo, float hi) {
    const quat diff = qnormalize(qmul(q2, qinv(q1)));
    const quat rel = qnormalize(qmul(diff, init_inv));
    const float c = rel.w;
    const float s = sqrtf(rel.x * rel.x + rel.y * rel.y + rel.z * rel.z);
    const float d = rel.x * a1.x + rel.y * a1.y + rel.z * a1.z;
    float angle = (d >= 0.0f) ? 2.0f * atan2f(s, c) : 2.0f * atan2f(s, -c);
    angle = hinge_normalized(angle);
    return hinge_near_limits(angle, lo, hi);
}

struct JBody {
    int32_t b;
    float im;
    v3 lf, af;
    bool dynamic;
};
RD JBody jbody(const DynArgs& a, int32_t b, bool dynamic) {
    JBody r;
    r.b = b;
    r.im = a.mass[b].y;
    r.lf = L3v(a.llock[b]);
    r.af = L3v(a.alock[b]);
    r.dynamic = dynamic;
    return r;
}

// --- fixed joint (SolveFixedJointSystem.cpp) ------------------------------
constexpr uint32_t JT_FIXED = 2, JT_SLIDER = 3;

// 3x3 rotation inverse mass: I1 + I2, inverted when its determinant is not
// tiny and a body is dynamic, else left as the sum (the reference keeps it).
RD M3 rotation_inverse_mass(const M3& I1, const M3& I2, bool dyn, bool* ok) {
    M3 K = m3_add(I1, I2);
    const float det = m3_det(K);
    *ok = fabsf(det) > MACHINE_EPSILON;
    if (*ok && dyn) K = m3_inverse(K, det);
    return K;
}
// 2 * (q2 * qinv0 * q1^-1).getVectorV() (SolveFixedJointSystem.cpp:419-421)
RD v3 rotation_error(quat q1, quat q2, float4 f0) {
    const quat e = qmul(qmul(q2, Q(f0.x, f0.y, f0.z, f0.w)), qinv(q1));
    return V(2.0f * e.x, 2.0f * e.y, 2.0f * e.z);
}

// initBeforeSolve (:49-133)
RD void fixed_init(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const int32_t b1 = e.y, b2 = e.z;
    const bool dyn = (e.w & 3) != 0;
    const M3 I1 = iiw_of(a, b1), I2 = iiw_of(a, b2);
    st3(q + JR_I1, I1);
    st3(q + JR_I2, I2);
    const float4 o1 = a.orientation[b1], o2 = a.orientation[b2];
    const quat q1 = Q(o1.x, o1.y, o1.z, o1.w), q2 = Q(o2.x, o2.y, o2.z, o2.w);
    const v3 r1 = qrot(q1, vsub(L3v(q[JR_LA1]), L3v(a.com_local[b1])));
    const v3 r2 = qrot(q2, vsub(L3v(q[JR_LA2]), L3v(a.com_local[b2])));
    q[JR_R1] = F4v(r1);
    q[JR_R2] = F4v(r2);
    const M3 K = joint_mass_matrix(a.mass[b1].y + a.mass[b2].y, m3_skew(r1), I1, m3_skew(r2), I2);
    M3 Kinv = m3_zero();
    const float det = m3_det(K);
    if (fabsf(det) > MACHINE_EPSILON && dyn) Kinv = m3_inverse(K, det);
    st3(q + JR_K, Kinv);
    bool ok;
    st3(q + JR_KR3, rotation_inverse_mass(I1, I2, dyn, &ok));
}

// warmstart (:136-186)
RD void fixed_warm(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const JBody B1 = jbody(a, e.y, false), B2 = jbody(a, e.z, false);
    v3 v1 = L3v(a.cv[e.y]), w1 = L3v(a.cw[e.y]), v2 = L3v(a.cv[e.z]), w2 = L3v(a.cw[e.z]);
    const M3 I1 = ld3(q + JR_I1), I2 = ld3(q + JR_I2);
    const v3 r1 = L3v(q[JR_R1]), r2 = L3v(q[JR_R2]);
    const v3 it = L3v(q[JR_IMP]), ir = L3v(q[JR_IMP2]);
    v3 ang1 = vcross(it, r1);
    ang1 = v3add(ang1, vneg(ir));
    v1 = v3add(v1, lin(B1.im, B1.lf, vneg(it)));
    w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, ang1)));
    v3 ang2 = vneg(vcross(it, r2));
    ang2 = v3add(ang2, ir);
    v2 = v3add(v2, lin(B2.im, B2.lf, it));
    w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, ang2)));
    a.cv[e.y] = F4v(v1); a.cw[e.y] = F4v(w1);
    a.cv[e.z] = F4v(v2); a.cw[e.z] = F4v(w2);
}

// solveVelocityConstraint (:189-262)
RD void fixed_solve(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const JBody B1 = jbody(a, e.y, false), B2 = jbody(a, e.z, false);
    v3 v1 = L3v(a.cv[e.y]), w1 = L3v(a.cw[e.y]), v2 = L3v(a.cv[e.z]), w2 = L3v(a.cw[e.z]);
    const M3 I1 = ld3(q + JR_I1), I2 = ld3(q + JR_I2);
    const v3 r1 = L3v(q[JR_R1]), r2 = L3v(q[JR_R2]);
    // translation: Jv = v2 + w2 x r2 - v1 - w1 x r1
    const v3 Jt = vsub(vsub(v3add(v2, vcross(w2, r2)), v1), vcross(w1, r1));
    const v3 dl = m3_mulv(ld3(q + JR_K), vsub(vneg(Jt), V(0.0f, 0.0f, 0.0f)));
    q[JR_IMP] = F4v(v3add(L3v(q[JR_IMP]), dl));
    v1 = v3add(v1, lin(B1.im, B1.lf, vneg(dl)));
    w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, vcross(dl, r1))));
    v2 = v3add(v2, lin(B2.im, B2.lf, dl));
    w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, vneg(vcross(dl, r2)))));
    // rotation: Jv = w2 - w1
    const v3 Jr = vsub(w2, w1);
    const v3 dr = m3_mulv(ld3(q + JR_KR3), vsub(vneg(Jr), V(0.0f, 0.0f, 0.0f)));
    q[JR_IMP2] = F4v(v3add(L3v(q[JR_IMP2]), dr));
    w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, vneg(dr))));
    w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, dr)));
    a.cv[e.y] = F4v(v1); a.cw[e.y] = F4v(w1);
    a.cv[e.z] = F4v(v2); a.cw[e.z] = F4v(w2);
}

// solvePositionConstraint, NON_LINEAR_GAUSS_SEIDEL (:265-447)
RD void fixed_position(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const bool dyn = (e.w & 3) != 0;
    const JBody B1 = jbody(a, e.y, false), B2 = jbody(a, e.z, false);
    const float4 t1 = a.qc[e.y], t2 = a.qc[e.z];
    quat q1 = Q(t1.x, t1.y, t1.z, t1.w), q2 = Q(t2.x, t2.y, t2.z, t2.w);
    float R[9];
    M3 I1, I2;
    quat_matrix(q1, R);
    world_inertia(R, L3v(a.iil[e.y]), I1.m);
    quat_matrix(q2, R);
    world_inertia(R, L3v(a.iil[e.z]), I2.m);
    st3(q + JR_I1, I1);
    st3(q + JR_I2, I2);
    const v3 r1 = qrot(q1, vsub(L3v(q[JR_LA1]), L3v(a.com_local[e.y])));
    const v3 r2 = qrot(q2, vsub(L3v(q[JR_LA2]), L3v(a.com_local[e.z])));
    q[JR_R1] = F4v(r1);
    q[JR_R2] = F4v(r2);
    v3 x1 = L3v(a.xc[e.y]), x2 = L3v(a.xc[e.z]);
    const M3 K = joint_mass_matrix(B1.im + B2.im, m3_skew(r1), I1, m3_skew(r2), I2);
    M3 Kinv = m3_zero();
    const float det = m3_det(K);
    if (fabsf(det) > MACHINE_EPSILON) {
        if (dyn) Kinv = m3_inverse(K, det);
        const v3 err = vsub(vsub(v3add(x2, r2), x1), r1);
        const v3 lam = m3_mulv(Kinv, vneg(err));
        x1 = v3add(x1, lin(B1.im, B1.lf, vneg(lam)));
        q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, vcross(lam, r1))));
        x2 = v3add(x2, lin(B2.im, B2.lf, lam));
        q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, vneg(vcross(lam, r2)))));
    }
    st3(q + JR_K, Kinv);
    bool ok;
    const M3 KR = rotation_inverse_mass(I1, I2, dyn, &ok);
    if (ok) {
        const v3 lam = m3_mulv(KR, vneg(rotation_error(q1, q2, q[JR_QINV])));
        q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, vneg(lam))));
        q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, lam)));
    }
    st3(q + JR_KR3, KR);
    a.xc[e.y] = F4v(x1);
    a.xc[e.z] = F4v(x2);
    a.qc[e.y] = make_float4(q1.x, q1.y, q1.z, q1.w);
    a.qc[e.z] = make_float4(q2.x, q2.y, q2.z, q2.w);
}

// --- slider joint (SolveSliderJointSystem.cpp) ----------------------------
RD v3 comb(float s, v3 a, float t, v3 b) {  // a * s + b * t
    return v3add(sv(s, a), sv(t, b));
}
RD v3 comb_neg(float s, v3 a, float t, v3 b) {  // -a * s - b * t
    return vsub(sv(s, vneg(a)), sv(t, b));
}
// el11 .. el22 of the 2x2 translation mass matrix and its inverse (zero when
// the determinant is tiny or no body is dynamic), :141-160 / :455-474.
RD float4 slider_translation_inverse(float sum_im, const M3& I1, const M3& I2, v3 r1n1, v3 r1n2, v3 r2n1, v3 r2n2,
                                     bool dyn, bool* ok) {
    const v3 i1n1 = m3_mulv(I1, r1n1), i1n2 = m3_mulv(I1, r1n2);
    const v3 i2n1 = m3_mulv(I2, r2n1), i2n2 = m3_mulv(I2, r2n2);
    const float e11 = sum_im + vdot(r1n1, i1n1) + vdot(r2n1, i2n1);
    const float e12 = vdot(r1n1, i1n2) + vdot(r2n1, i2n2);
    const float e21 = vdot(r1n2, i1n1) + vdot(r2n2, i2n1);
    const float e22 = sum_im + vdot(r1n2, i1n2) + vdot(r2n2, i2n2);
    const float d = e11 * e22 - e21 * e12;
    *ok = fabsf(d) > MACHINE_EPSILON;
    if (*ok && dyn) {
        const float inv = 1.0f / d;
        return make_float4(e22 * inv, -e12 * inv, -e21 * inv, e11 * inv);
    }
    return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
// 1 / (im1 + im2 + (r1+u)xa . I1 (r1+u)xa + r2xa . I2 r2xa), or 0
RD float slider_limit_inverse(float im1, float im2, const M3& I1, const M3& I2, v3 r1a, v3 r2a) {
    float k = im1 + im2 + vdot(r1a, m3_mulv(I1, r1a)) + vdot(r2a, m3_mulv(I2, r2a));
    return (k > 0.0f) ? 1.0f / k : 0.0f;
}

// initBeforeSolve (:49-170).  The limit's inverse mass is computed from the
// r2 x axis row before this step's value replaces it (the reference reads
// mR2CrossSliderAxis ahead of its update).
RD void slider_init(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const int32_t b1 = e.y, b2 = e.z;
    const bool dyn = (e.w & 3) != 0;
    const uint32_t flags = uint32_t(__float_as_int(q[JR_HDR].y));
    const M3 I1 = iiw_of(a, b1), I2 = iiw_of(a, b2);
    st3(q + JR_I1, I1);
    st3(q + JR_I2, I2);
    const float4 o1 = a.orientation[b1], o2 = a.orientation[b2];
    const quat q1 = Q(o1.x, o1.y, o1.z, o1.w), q2 = Q(o2.x, o2.y, o2.z, o2.w);
    const v3 r1 = qrot(q1, vsub(L3v(q[JR_LA1]), L3v(a.com_local[b1])));
    const v3 r2 = qrot(q2, vsub(L3v(q[JR_LA2]), L3v(a.com_local[b2])));
    q[JR_R1] = F4v(r1);
    q[JR_R2] = F4v(r2);
    const v3 ax = vnormalize(qrot(q1, L3v(q[JR_AX1])));
    const v3 n1 = unit_orthogonal(ax);
    const v3 n2 = vcross(ax, n1);
    const v3 x1 = L3v(a.com_world[b1]), x2 = L3v(a.com_world[b2]);
    const v3 u = vsub(vsub(v3add(x2, r2), x1), r1);
    const v3 r1u = v3add(r1, u);
    const v3 r1n1 = vcross(r1u, n1), r1n2 = vcross(r1u, n2), r1a = vcross(r1u, ax);
    const float4 par = q[JR_PARAM];
    const float ud = vdot(u, ax);
    const float lerr = ud - par.y, uerr = par.z - ud;
    float4 st = q[JR_STATE], imp = q[JR_IMP], misc = q[JR_MISC];
    const bool oldl = st.x != 0.0f, lv = lerr <= 0.0f;
    st.x = lv ? 1.0f : 0.0f;
    if (!lv || lv != oldl) imp.z = 0.0f;
    const bool oldu = st.y != 0.0f, uv = uerr <= 0.0f;
    st.y = uv ? 1.0f : 0.0f;
    if (!uv || uv != oldu) imp.w = 0.0f;
    const float im1 = a.mass[b1].y, im2 = a.mass[b2].y;
    if ((flags & JF_LIMIT) && (lv || uv)) misc.x = slider_limit_inverse(im1, im2, I1, I2, r1a, L3v(q[JR_R2A]));
    const v3 r2n1 = vcross(r2, n1), r2n2 = vcross(r2, n2), r2a = vcross(r2, ax);
    bool ok;
    q[JR_KROT] = slider_translation_inverse(im1 + im2, I1, I2, r1n1, r1n2, r2n1, r2n2, dyn, &ok);
    st3(q + JR_KR3, rotation_inverse_mass(I1, I2, dyn, &ok));
    if (flags & JF_MOTOR) {
        const float s = im1 + im2;
        misc.y = (s > 0.0f) ? 1.0f / s : 0.0f;
    }
    q[JR_A1] = F4v(ax);
    q[JR_N1] = F4v(n1);
    q[JR_N2] = F4v(n2);
    q[JR_R1N1] = F4v(r1n1);
    q[JR_R1N2] = F4v(r1n2);
    q[JR_R1A] = F4v(r1a);
    q[JR_R2N1] = F4v(r2n1);
    q[JR_R2N2] = F4v(r2n2);
    q[JR_R2A] = F4v(r2a);
    q[JR_STATE] = st;
    q[JR_IMP] = imp;
    q[JR_MISC] = misc;
}

// warmstart (:173-248)
RD void slider_warm(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const JBody B1 = jbody(a, e.y, false), B2 = jbody(a, e.z, false);
    v3 v1 = L3v(a.cv[e.y]), w1 = L3v(a.cw[e.y]), v2 = L3v(a.cv[e.z]), w2 = L3v(a.cw[e.z]);
    const M3 I1 = ld3(q + JR_I1), I2 = ld3(q + JR_I2);
    const v3 ax = L3v(q[JR_A1]), n1 = L3v(q[JR_N1]), n2 = L3v(q[JR_N2]);
    const float4 imp = q[JR_IMP];
    const v3 ir = L3v(q[JR_IMP2]);
    const float il = imp.w - imp.z;
    const v3 lim = sv(il, ax);
    const v3 mot = sv(q[JR_STATE].z, ax);
    v3 lin1 = comb_neg(imp.x, n1, imp.y, n2);
    v3 ang1 = comb_neg(imp.x, L3v(q[JR_R1N1]), imp.y, L3v(q[JR_R1N2]));
    ang1 = v3add(ang1, vneg(ir));
    lin1 = v3add(lin1, lim);
    ang1 = v3add(ang1, sv(il, L3v(q[JR_R1A])));
    lin1 = v3add(lin1, mot);
    v1 = v3add(v1, lin(B1.im, B1.lf, lin1));
    w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, ang1)));
    v3 lin2 = comb(imp.x, n1, imp.y, n2);
    v3 ang2 = comb(imp.x, L3v(q[JR_R2N1]), imp.y, L3v(q[JR_R2N2]));
    ang2 = v3add(ang2, ir);
    lin2 = v3add(lin2, vneg(lim));
    ang2 = v3add(ang2, sv(-il, L3v(q[JR_R2A])));
    lin2 = v3add(lin2, vneg(mot));
    v2 = v3add(v2, lin(B2.im, B2.lf, lin2));
    w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, ang2)));
    a.cv[e.y] = F4v(v1); a.cw[e.y] = F4v(w1);
    a.cv[e.z] = F4v(v2); a.cw[e.z] = F4v(w2);
}

// solveVelocityConstraint (:251-415)
RD void slider_solve(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const uint32_t flags = uint32_t(__float_as_int(q[JR_HDR].y));
    const JBody B1 = jbody(a, e.y, false), B2 = jbody(a, e.z, false);
    v3 v1 = L3v(a.cv[e.y]), w1 = L3v(a.cw[e.y]), v2 = L3v(a.cv[e.z]), w2 = L3v(a.cw[e.z]);
    const M3 I1 = ld3(q + JR_I1), I2 = ld3(q + JR_I2);
    const v3 ax = L3v(q[JR_A1]), n1 = L3v(q[JR_N1]), n2 = L3v(q[JR_N2]);
    const v3 r2n1 = L3v(q[JR_R2N1]), r2n2 = L3v(q[JR_R2N2]), r2a = L3v(q[JR_R2A]);
    const v3 r1n1 = L3v(q[JR_R1N1]), r1n2 = L3v(q[JR_R1N2]), r1a = L3v(q[JR_R1A]);
    float4 imp = q[JR_IMP], st = q[JR_STATE];
    const float4 misc = q[JR_MISC];
    if (flags & JF_LIMIT) {
        if (st.x != 0.0f) {
            const float Jv = vdot(ax, v2) + vdot(r2a, w2) - vdot(ax, v1) - vdot(r1a, w1);
            float dl = misc.x * (-Jv - 0.0f);
            const float lt = imp.z;
            imp.z = smax(imp.z + dl, 0.0f);
            dl = imp.z - lt;
            v1 = v3add(v1, lin(B1.im, B1.lf, sv(-dl, ax)));
            w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, sv(-dl, r1a))));
            v2 = v3add(v2, lin(B2.im, B2.lf, sv(dl, ax)));
            w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, sv(dl, r2a))));
        }
        if (st.y != 0.0f) {
            const float Jv = vdot(ax, v1) + vdot(r1a, w1) - vdot(ax, v2) - vdot(r2a, w2);
            float dl = misc.x * (-Jv - 0.0f);
            const float lt = imp.w;
            imp.w = smax(imp.w + dl, 0.0f);
            dl = imp.w - lt;
            v1 = v3add(v1, lin(B1.im, B1.lf, sv(dl, ax)));
            w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, sv(dl, r1a))));
            v2 = v3add(v2, lin(B2.im, B2.lf, sv(-dl, ax)));
            w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, sv(-dl, r2a))));
        }
    }
    if (flags & JF_MOTOR) {
        const float Jv = vdot(ax, v1) - vdot(ax, v2);
        const float maxi = q[JR_PARAM2].x * a.dt;
        float dl = misc.y * (-Jv - q[JR_PARAM].w);
        const float lt = st.z;
        st.z = sclamp(st.z + dl, -maxi, maxi);
        dl = st.z - lt;
        v1 = v3add(v1, lin(B1.im, B1.lf, sv(dl, ax)));
        v2 = v3add(v2, lin(B2.im, B2.lf, sv(-dl, ax)));
    }
    // rotation: Jv = w2 - w1
    const v3 dr = m3_mulv(ld3(q + JR_KR3), vsub(vneg(vsub(w2, w1)), V(0.0f, 0.0f, 0.0f)));
    q[JR_IMP2] = F4v(v3add(L3v(q[JR_IMP2]), dr));
    w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, vneg(dr))));
    w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, dr)));
    // translation along n1, n2
    const float el1 = -vdot(n1, v1) - vdot(w1, r1n1) + vdot(n1, v2) + vdot(w2, r2n1);
    const float el2 = -vdot(n2, v1) - vdot(w1, r1n2) + vdot(n2, v2) + vdot(w2, r2n2);
    const float4 kt = q[JR_KROT];
    const float rx = -el1 - 0.0f, ry = -el2 - 0.0f;
    const float dx = kt.x * rx + kt.y * ry, dy = kt.z * rx + kt.w * ry;
    imp.x = imp.x + dx;
    imp.y = imp.y + dy;
    const v3 lin1 = comb_neg(dx, n1, dy, n2);
    v1 = v3add(v1, lin(B1.im, B1.lf, lin1));
    w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, comb_neg(dx, r1n1, dy, r1n2))));
    v2 = v3add(v2, lin(B2.im, B2.lf, vneg(lin1)));
    w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, comb(dx, r2n1, dy, r2n2))));
    q[JR_IMP] = imp;
    q[JR_STATE] = st;
    a.cv[e.y] = F4v(v1); a.cw[e.y] = F4v(w1);
    a.cv[e.z] = F4v(v2); a.cw[e.z] = F4v(w2);
}

// solvePositionConstraint, NON_LINEAR_GAUSS_SEIDEL (:418-596).  The
// translation error is the one measured before the limit corrections.
RD void slider_position(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const uint32_t flags = uint32_t(__float_as_int(q[JR_HDR].y));
    const bool dyn = (e.w & 3) != 0;
    const JBody B1 = jbody(a, e.y, false), B2 = jbody(a, e.z, false);
    const float4 t1 = a.qc[e.y], t2 = a.qc[e.z];
    quat q1 = Q(t1.x, t1.y, t1.z, t1.w), q2 = Q(t2.x, t2.y, t2.z, t2.w);
    float R[9];
    M3 I1, I2;
    quat_matrix(q1, R);
    world_inertia(R, L3v(a.iil[e.y]), I1.m);
    quat_matrix(q2, R);
    world_inertia(R, L3v(a.iil[e.z]), I2.m);
    st3(q + JR_I1, I1);
    st3(q + JR_I2, I2);
    const v3 r1 = qrot(q1, vsub(L3v(q[JR_LA1]), L3v(a.com_local[e.y])));
    const v3 r2 = qrot(q2, vsub(L3v(q[JR_LA2]), L3v(a.com_local[e.z])));
    q[JR_R1] = F4v(r1);
    q[JR_R2] = F4v(r2);
    v3 x1 = L3v(a.xc[e.y]), x2 = L3v(a.xc[e.z]);
    const v3 u = vsub(vsub(v3add(x2, r2), x1), r1);
    const v3 ax = vnormalize(qrot(q1, L3v(q[JR_AX1])));
    const v3 n1 = unit_orthogonal(ax);
    const v3 n2 = vcross(ax, n1);
    const float4 par = q[JR_PARAM];
    const float ud = vdot(u, ax);
    float4 st = q[JR_STATE], misc = q[JR_MISC];
    st.x = (ud - par.y <= 0.0f) ? 1.0f : 0.0f;
    st.y = (par.z - ud <= 0.0f) ? 1.0f : 0.0f;
    const v3 r2n1 = vcross(r2, n1), r2n2 = vcross(r2, n2), r2a = vcross(r2, ax);
    const v3 r1u = v3add(r1, u);
    const v3 r1n1 = vcross(r1u, n1), r1n2 = vcross(r1u, n2), r1a = vcross(r1u, ax);
    if (flags & JF_LIMIT) {
        if (st.x != 0.0f || st.y != 0.0f) misc.x = slider_limit_inverse(B1.im, B2.im, I1, I2, r1a, r2a);
        if (st.x != 0.0f) {
            const v3 uu = vsub(vsub(v3add(x2, r2), x1), r1);
            const float lam = misc.x * (-(vdot(uu, ax) - par.y));
            x1 = v3add(x1, lin(B1.im, B1.lf, sv(-lam, ax)));
            q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, sv(-lam, r1a))));
            x2 = v3add(x2, lin(B2.im, B2.lf, sv(lam, ax)));
            q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, sv(lam, r2a))));
        }
        if (st.y != 0.0f) {
            const v3 uu = vsub(vsub(v3add(x2, r2), x1), r1);
            const float lam = misc.x * (-(par.z - vdot(uu, ax)));
            x1 = v3add(x1, lin(B1.im, B1.lf, sv(lam, ax)));
            q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, sv(lam, r1a))));
            x2 = v3add(x2, lin(B2.im, B2.lf, sv(-lam, ax)));
            q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, sv(-lam, r2a))));
        }
    }
    bool ok;
    const M3 KR = rotation_inverse_mass(I1, I2, dyn, &ok);
    if (ok) {
        const v3 lam = m3_mulv(KR, vneg(rotation_error(q1, q2, q[JR_QINV])));
        q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, vneg(lam))));
        q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, lam)));
    }
    st3(q + JR_KR3, KR);
    const float4 kt = slider_translation_inverse(B1.im + B2.im, I1, I2, r1n1, r1n2, r2n1, r2n2, dyn, &ok);
    if (ok) {
        const float ex = -vdot(u, n1), ey = -vdot(u, n2);
        const float lx = kt.x * ex + kt.y * ey, ly = kt.z * ex + kt.w * ey;
        x1 = v3add(x1, lin(B1.im, B1.lf, comb_neg(lx, n1, ly, n2)));
        q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, comb_neg(lx, r1n1, ly, r1n2))));
        x2 = v3add(x2, lin(B2.im, B2.lf, comb(lx, n1, ly, n2)));
        q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, comb(lx, r2n1, ly, r2n2))));
    }
    q[JR_KROT] = kt;
    q[JR_A1] = F4v(ax);
    q[JR_N1] = F4v(n1);
    q[JR_N2] = F4v(n2);
    q[JR_R1N1] = F4v(r1n1);
    q[JR_R1N2] = F4v(r1n2);
    q[JR_R1A] = F4v(r1a);
    q[JR_R2N1] = F4v(r2n1);
    q[JR_R2N2] = F4v(r2n2);
    q[JR_R2A] = F4v(r2a);
    q[JR_STATE] = st;
    q[JR_MISC] = misc;
    a.xc[e.y] = F4v(x1);
    a.xc[e.z] = F4v(x2);
    a.qc[e.y] = make_float4(q1.x, q1.y, q1.z, q1.w);
    a.qc[e.z] = make_float4(q2.x, q2.y, q2.z, q2.w);
}

// initBeforeSolve of one joint (BallAndSocket :49-136, Hinge :48-214).
RD void joint_init(const DynArgs& a, const int4 e) {
    JointRec* R = a.j_rec + e.x;
    float4* q = R->q;
    const uint32_t jt = uint32_t(__float_as_int(q[JR_HDR].x));
    if (jt == JT_FIXED) return fixed_init(a, e);
    if (jt == JT_SLIDER) return slider_init(a, e);
    const int32_t b1 = e.y, b2 = e.z;
    const bool dyn1 = (e.w & 1) != 0, dyn2 = (e.w & 2) != 0;
    const uint32_t type = uint32_t(__float_as_int(q[JR_HDR].x));
    const uint32_t flags = uint32_t(__float_as_int(q[JR_HDR].y));
    const M3 I1 = iiw_of(a, b1), I2 = iiw_of(a, b2);
    st3(q + JR_I1, I1);
    st3(q + JR_I2, I2);
    const float4 o1 = a.orientation[b1], o2 = a.orientation[b2];
    const quat q1 = Q(o1.x, o1.y, o1.z, o1.w), q2 = Q(o2.x, o2.y, o2.z, o2.w);
    const v3 r1 = qrot(q1, vsub(L3v(q[JR_LA1]), L3v(a.com_local[b1])));
    const v3 r2 = qrot(q2, vsub(L3v(q[JR_LA2]), L3v(a.com_local[b2])));
    q[JR_R1] = F4v(r1);
    q[JR_R2] = F4v(r2);
    const M3 U1 = m3_skew(r1), U2 = m3_skew(r2);
    const float im1 = a.mass[b1].y, im2 = a.mass[b2].y;
    const M3 K = joint_mass_matrix(im1 + im2, U1, I1, U2, I2);
    M3 Kinv = m3_zero();
    const float det = m3_det(K);
    if (fabsf(det) > MACHINE_EPSILON && (dyn1 || dyn2)) Kinv = m3_inverse(K, det);
    st3(q + JR_K, Kinv);
    float4 st = q[JR_STATE];  // ball-socket: cone impulse, cone violated; hinge: lower / upper violated, motor impulse
    float4 imp2 = q[JR_IMP2];
    if (type == 0) {
        const v3 u1 = vunit(r1), u2 = vunit(r2);
        const v3 nu2 = vneg(u2);
        const v3 acb = vcross(u1, nu2);
        q[JR_ACB] = F4v(acb);
        const float cone = acosf(vdot(u1, nu2));
        const float err = q[JR_PARAM].x - cone;
        const bool old = st.y != 0.0f;
        const bool viol = err < 0.0f;
        st.y = viol ? 1.0f : 0.0f;
        if (!viol || viol != old) st.x = 0.0f;
        if (flags & JF_CONE) {
            float im = vdot(acb, m3_mulv(I1, acb)) + vdot(acb, m3_mulv(I2, acb));
            im = (im > 0.0f) ? 1.0f / im : 0.0f;
            q[JR_MISC] = make_float4(im, 0.0f, 0.0f, 0.0f);
        }
    } else {
        v3 a1 = vnormalize(qrot(q1, L3v(q[JR_AX1])));
        v3 a2 = vnormalize(qrot(q2, L3v(q[JR_AX2])));
        const v3 b2 = unit_orthogonal(a2);
        const v3 c2 = vcross(a2, b2);
        const v3 b2a1 = vcross(b2, a1), c2a1 = vcross(c2, a1);
        q[JR_A1] = F4v(a1);
        q[JR_B2A1] = F4v(b2a1);
        q[JR_C2A1] = F4v(c2a1);
        const v3 i1b = m3_mulv(I1, b2a1), i1c = m3_mulv(I1, c2a1), i2b = m3_mulv(I2, b2a1), i2c = m3_mulv(I2, c2a1);
        const float e11 = vdot(b2a1, i1b) + vdot(b2a1, i2b);
        const float e12 = vdot(b2a1, i1c) + vdot(b2a1, i2c);
        const float e21 = vdot(c2a1, i1b) + vdot(c2a1, i2b);
        const float e22 = vdot(c2a1, i1c) + vdot(c2a1, i2c);
        float4 kr = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float d2 = e11 * e22 - e21 * e12;
        if (fabsf(d2) > MACHINE_EPSILON && (dyn1 || dyn2)) {
            const float inv = 1.0f / d2;
            kr = make_float4(e22 * inv, -e12 * inv, -e21 * inv, e11 * inv);
        }
        q[JR_KROT] = kr;
        const float4 par = q[JR_PARAM];  // x unused, y lower, z upper, w motor speed
        const float4 f0 = q[JR_QINV];
        const float angle = hinge_angle(q1, q2, Q(f0.x, f0.y, f0.z, f0.w), a1, par.y, par.z);
        const float lerr = angle - par.y, uerr = par.z - angle;
        const bool oldl = st.x != 0.0f, lv = lerr <= 0.0f;
        st.x = lv ? 1.0f : 0.0f;
        if (!lv || lv != oldl) imp2.z = 0.0f;
        const bool oldu = st.y != 0.0f, uv = uerr <= 0.0f;
        st.y = uv ? 1.0f : 0.0f;
        if (!uv || uv != oldu) imp2.w = 0.0f;
        if ((flags & JF_MOTOR) || ((flags & JF_LIMIT) && (lv || uv))) {
            float im = vdot(a1, m3_mulv(I1, a1)) + vdot(a1, m3_mulv(I2, a1));
            im = (im > 0.0f) ? 1.0f / im : 0.0f;
            float4 misc = q[JR_MISC];
            misc.x = im;
            q[JR_MISC] = misc;
        }
    }
    q[JR_STATE] = st;
    q[JR_IMP2] = imp2;
}

// warmstart of one joint (BallAndSocket :139-197, Hinge :217-297).
RD void joint_warm(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const uint32_t type = uint32_t(__float_as_int(q[JR_HDR].x));
    if (type == JT_FIXED) return fixed_warm(a, e);
    if (type == JT_SLIDER) return slider_warm(a, e);
    const JBody B1 = jbody(a, e.y, false), B2 = jbody(a, e.z, false);
    v3 v1 = L3v(a.cv[e.y]), w1 = L3v(a.cw[e.y]), v2 = L3v(a.cv[e.z]), w2 = L3v(a.cw[e.z]);
    const M3 I1 = ld3(q + JR_I1), I2 = ld3(q + JR_I2);
    const v3 r1 = L3v(q[JR_R1]), r2 = L3v(q[JR_R2]);
    const v3 imp = L3v(q[JR_IMP]);
    if (type == 0) {
        const v3 lin1 = vneg(imp);
        v3 ang1 = vcross(imp, r1);
        const v3 cone = sv(q[JR_STATE].x, L3v(q[JR_ACB]));
        ang1 = v3add(ang1, cone);
        v1 = v3add(v1, lin(B1.im, B1.lf, lin1));
        w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, ang1)));
        v3 ang2 = vneg(vcross(imp, r2));
        ang2 = v3add(ang2, vneg(cone));
        v2 = v3add(v2, lin(B2.im, B2.lf, imp));
        w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, ang2)));
    } else {
        const float4 imp2 = q[JR_IMP2];  // rotation x, y, lower, upper
        const v3 b2a1 = L3v(q[JR_B2A1]), c2a1 = L3v(q[JR_C2A1]), a1 = L3v(q[JR_A1]);
        // -b2CrossA1 * x - c2CrossA1 * y
        const v3 nb = vneg(b2a1);
        const v3 rot = vsub(V(nb.x * imp2.x, nb.y * imp2.x, nb.z * imp2.x), V(c2a1.x * imp2.y, c2a1.y * imp2.y, c2a1.z * imp2.y));
        const v3 lim = sv(imp2.w - imp2.z, a1);
        const v3 mot = sv(-q[JR_STATE].z, a1);
        const v3 lin1 = vneg(imp);
        v3 ang1 = vcross(imp, r1);
        ang1 = v3add(ang1, rot);
        ang1 = v3add(ang1, lim);
        ang1 = v3add(ang1, mot);
        v1 = v3add(v1, lin(B1.im, B1.lf, lin1));
        w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, ang1)));
        v3 ang2 = vneg(vcross(imp, r2));
        ang2 = v3add(ang2, vneg(rot));
        ang2 = v3add(ang2, vneg(lim));
        ang2 = v3add(ang2, vneg(mot));
        v2 = v3add(v2, lin(B2.im, B2.lf, imp));
        w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, ang2)));
    }
    a.cv[e.y] = F4v(v1); a.cw[e.y] = F4v(w1);
    a.cv[e.z] = F4v(v2); a.cw[e.z] = F4v(w2);
}

// solveVelocityConstraint of one joint (BallAndSocket :200-295, Hinge :300-471).
RD void joint_solve(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const uint32_t type = uint32_t(__float_as_int(q[JR_HDR].x));
    if (type == JT_FIXED) return fixed_solve(a, e);
    if (type == JT_SLIDER) return slider_solve(a, e);
    const uint32_t flags = uint32_t(__float_as_int(q[JR_HDR].y));
    const JBody B1 = jbody(a, e.y, false), B2 = jbody(a, e.z, false);
    v3 v1 = L3v(a.cv[e.y]), w1 = L3v(a.cw[e.y]), v2 = L3v(a.cv[e.z]), w2 = L3v(a.cw[e.z]);
    const M3 I1 = ld3(q + JR_I1), I2 = ld3(q + JR_I2);
    const v3 r1 = L3v(q[JR_R1]), r2 = L3v(q[JR_R2]);
    float4 st = q[JR_STATE];
    if (type == 0) {
        if ((flags & JF_CONE) && st.y != 0.0f) {
            const v3 acb = L3v(q[JR_ACB]);
            const float Jv = vdot(acb, vsub(w1, w2));
            float dl = q[JR_MISC].x * (-Jv - 0.0f);
            const float lt = st.x;
            st.x = smax(st.x + dl, 0.0f);
            dl = st.x - lt;
            w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, sv(dl, acb))));
            w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, sv(-dl, acb))));
        }
        // Jv = v2 + w2 x r2 - v1 - w1 x r1
        const v3 Jv = vsub(vsub(v3add(v2, vcross(w2, r2)), v1), vcross(w1, r1));
        const M3 K = ld3(q + JR_K);
        const v3 rhs = vsub(vneg(Jv), V(0.0f, 0.0f, 0.0f));
        const v3 dl = m3_mulv(K, rhs);
        q[JR_IMP] = F4v(v3add(L3v(q[JR_IMP]), dl));
        v1 = v3add(v1, lin(B1.im, B1.lf, vneg(dl)));
        w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, vcross(dl, r1))));
        w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, vneg(vcross(dl, r2)))));
        v2 = v3add(v2, lin(B2.im, B2.lf, dl));
    } else {
        const v3 a1 = L3v(q[JR_A1]);
        const float imm = q[JR_MISC].x;
        float4 imp2 = q[JR_IMP2];
        if (flags & JF_LIMIT) {
            if (st.x != 0.0f) {
                const float Jv = vdot(vsub(w2, w1), a1);
                float dl = imm * (-Jv - 0.0f);
                const float lt = imp2.z;
                imp2.z = smax(imp2.z + dl, 0.0f);
                dl = imp2.z - lt;
                w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, sv(-dl, a1))));
                w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, sv(dl, a1))));
            }
            if (st.y != 0.0f) {
                const float Jv = -vdot(vsub(w2, w1), a1);
                float dl = imm * (-Jv - 0.0f);
                const float lt = imp2.w;
                imp2.w = smax(imp2.w + dl, 0.0f);
                dl = imp2.w - lt;
                w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, sv(dl, a1))));
                w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, sv(-dl, a1))));
            }
        }
        if (flags & JF_MOTOR) {
            const float Jv = vdot(a1, vsub(w1, w2));
            const float maxi = q[JR_PARAM2].x * a.dt;
            float dl = imm * (-Jv - q[JR_PARAM].w);
            const float lt = st.z;
            st.z = sclamp(st.z + dl, -maxi, maxi);
            dl = st.z - lt;
            w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, sv(-dl, a1))));
            w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, sv(dl, a1))));
        }
        const v3 b2a1 = L3v(q[JR_B2A1]), c2a1 = L3v(q[JR_C2A1]);
        const float jr0 = -vdot(b2a1, w1) + vdot(b2a1, w2);
        const float jr1 = -vdot(c2a1, w1) + vdot(c2a1, w2);
        const float4 kr = q[JR_KROT];
        const float rx = -jr0 - 0.0f, ry = -jr1 - 0.0f;
        const float dx = kr.x * rx + kr.y * ry, dy = kr.z * rx + kr.w * ry;
        imp2.x = imp2.x + dx;
        imp2.y = imp2.y + dy;
        const v3 nb = vneg(b2a1);
        v3 ang1 = vsub(V(nb.x * dx, nb.y * dx, nb.z * dx), V(c2a1.x * dy, c2a1.y * dy, c2a1.z * dy));
        w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, ang1)));
        v3 ang2 = v3add(V(b2a1.x * dx, b2a1.y * dx, b2a1.z * dx), V(c2a1.x * dy, c2a1.y * dy, c2a1.z * dy));
        w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, ang2)));
        const v3 Jt = vsub(vsub(v3add(v2, vcross(w2, r2)), v1), vcross(w1, r1));
        const M3 K = ld3(q + JR_K);
        const v3 dl = m3_mulv(K, vsub(vneg(Jt), V(0.0f, 0.0f, 0.0f)));
        q[JR_IMP] = F4v(v3add(L3v(q[JR_IMP]), dl));
        ang1 = vcross(dl, r1);
        v1 = v3add(v1, lin(B1.im, B1.lf, vneg(dl)));
        w1 = v3add(w1, vcmul(B1.af, m3_mulv(I1, ang1)));
        ang2 = vneg(vcross(dl, r2));
        v2 = v3add(v2, lin(B2.im, B2.lf, dl));
        w2 = v3add(w2, vcmul(B2.af, m3_mulv(I2, ang2)));
        q[JR_IMP2] = imp2;
    }
    q[JR_STATE] = st;
    a.cv[e.y] = F4v(v1); a.cw[e.y] = F4v(w1);
    a.cv[e.z] = F4v(v2); a.cw[e.z] = F4v(w2);
}

// solvePositionConstraint of one joint, NON_LINEAR_GAUSS_SEIDEL
// (BallAndSocket :298-445, Hinge :474-716), on the constrained positions and
// orientations (a.xc, a.qc).
RD void joint_position(const DynArgs& a, const int4 e) {
    float4* q = a.j_rec[e.x].q;
    const uint32_t type = uint32_t(__float_as_int(q[JR_HDR].x));
    if (type == JT_FIXED) return fixed_position(a, e);
    if (type == JT_SLIDER) return slider_position(a, e);
    const uint32_t flags = uint32_t(__float_as_int(q[JR_HDR].y));
    const bool dyn1 = (e.w & 1) != 0, dyn2 = (e.w & 2) != 0;
    const JBody B1 = jbody(a, e.y, dyn1), B2 = jbody(a, e.z, dyn2);
    float4 t1 = a.qc[e.y], t2 = a.qc[e.z];
    quat q1 = Q(t1.x, t1.y, t1.z, t1.w), q2 = Q(t2.x, t2.y, t2.z, t2.w);
    float R[9];
    M3 I1, I2;
    quat_matrix(q1, R);
    world_inertia(R, L3v(a.iil[e.y]), I1.m);
    quat_matrix(q2, R);
    world_inertia(R, L3v(a.iil[e.z]), I2.m);
    st3(q + JR_I1, I1);
    st3(q + JR_I2, I2);
    v3 r1 = qrot(q1, vsub(L3v(q[JR_LA1]), L3v(a.com_local[e.y])));
    v3 r2 = qrot(q2, vsub(L3v(q[JR_LA2]), L3v(a.com_local[e.z])));
    q[JR_R1] = F4v(r1);
    q[JR_R2] = F4v(r2);
    const M3 U1 = m3_skew(r1), U2 = m3_skew(r2);
    const float im1 = B1.im, im2 = B2.im;
    v3 x1 = L3v(a.xc[e.y]), x2 = L3v(a.xc[e.z]);
    float4 st = q[JR_STATE];
    if (type == 0) {
        if (flags & JF_CONE) {
            const v3 u1 = vunit(r1), u2 = vunit(r2);
            const v3 nu2 = vneg(u2);
            const v3 acb = vcross(u1, nu2);
            q[JR_ACB] = F4v(acb);
            const float cone = acosf(vdot(u1, nu2));
            const float err = q[JR_PARAM].x - cone;
            st.y = (err < 0.0f) ? 1.0f : 0.0f;
            if (st.y != 0.0f) {
                float im = vdot(acb, m3_mulv(I1, acb)) + vdot(acb, m3_mulv(I2, acb));
                im = (im > 0.0f) ? 1.0f / im : 0.0f;
                float4 misc = q[JR_MISC];
                misc.x = im;
                q[JR_MISC] = misc;
                const float lam = im * (-err);
                q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, sv(lam, acb))));
                q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, sv(-lam, acb))));
            }
        }
        const M3 K = joint_mass_matrix(im1 + im2, U1, I1, U2, I2);
        M3 Kinv = m3_zero();
        const float det = m3_det(K);
        if (fabsf(det) > MACHINE_EPSILON) {
            if (dyn1 || dyn2) Kinv = m3_inverse(K, det);
            // x2 + r2World - x1 - r1World
            const v3 err = vsub(vsub(v3add(x2, r2), x1), r1);
            const v3 lam = m3_mulv(Kinv, vneg(err));
            x1 = v3add(x1, lin(im1, B1.lf, vneg(lam)));
            q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, vcross(lam, r1))));
            x2 = v3add(x2, lin(im2, B2.lf, lam));
            q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, vneg(vcross(lam, r2)))));
        }
        st3(q + JR_K, Kinv);
    } else {
        v3 a1 = vnormalize(qrot(q1, L3v(q[JR_AX1])));
        v3 a2 = vnormalize(qrot(q2, L3v(q[JR_AX2])));
        const v3 b2 = unit_orthogonal(a2);
        const v3 c2 = vcross(a2, b2);
        const v3 b2a1 = vcross(b2, a1), c2a1 = vcross(c2, a1);
        q[JR_A1] = F4v(a1);
        q[JR_B2A1] = F4v(b2a1);
        q[JR_C2A1] = F4v(c2a1);
        const float4 par = q[JR_PARAM];
        const float4 f0 = q[JR_QINV];
        const float angle = hinge_angle(q1, q2, Q(f0.x, f0.y, f0.z, f0.w), a1, par.y, par.z);
        const float lerr = angle - par.y, uerr = par.z - angle;
        st.x = (lerr <= 0.0f) ? 1.0f : 0.0f;
        st.y = (uerr <= 0.0f) ? 1.0f : 0.0f;
        if (flags & JF_LIMIT) {
            float4 misc = q[JR_MISC];
            const float imm = misc.x;   // the value before this update is the one used below
            if (st.x != 0.0f || st.y != 0.0f) {
                const float k = vdot(a1, m3_mulv(I1, a1)) + vdot(a1, m3_mulv(I2, a1));
                misc.x = (imm > 0.0f) ? 1.0f / k : 0.0f;
                q[JR_MISC] = misc;
            }
            if (st.x != 0.0f) {
                const float lam = imm * (-lerr);
                q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, sv(-lam, a1))));
                q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, sv(lam, a1))));
            }
            if (st.y != 0.0f) {
                const float lam = imm * (-uerr);
                q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, sv(lam, a1))));
                q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, sv(-lam, a1))));
            }
        }
        const v3 i1b = m3_mulv(I1, b2a1), i1c = m3_mulv(I1, c2a1), i2b = m3_mulv(I2, b2a1), i2c = m3_mulv(I2, c2a1);
        const float e11 = vdot(b2a1, i1b) + vdot(b2a1, i2b);
        const float e12 = vdot(b2a1, i1c) + vdot(b2a1, i2c);
        const float e21 = vdot(c2a1, i1b) + vdot(c2a1, i2b);
        const float e22 = vdot(c2a1, i1c) + vdot(c2a1, i2c);
        float4 kr = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float d2 = e11 * e22 - e21 * e12;
        if (fabsf(d2) > MACHINE_EPSILON) {
            if (dyn1 || dyn2) {
                const float inv = 1.0f / d2;
                kr = make_float4(e22 * inv, -e12 * inv, -e21 * inv, e11 * inv);
            }
            const float ex = vdot(a1, b2), ey = vdot(a1, c2);
            const float rx = -ex, ry = -ey;
            const float lx = kr.x * rx + kr.y * ry, ly = kr.z * rx + kr.w * ry;
            const v3 nb = vneg(b2a1);
            const v3 ang1 = vsub(V(nb.x * lx, nb.y * lx, nb.z * lx), V(c2a1.x * ly, c2a1.y * ly, c2a1.z * ly));
            q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, ang1)));
            const v3 ang2 = v3add(V(b2a1.x * lx, b2a1.y * lx, b2a1.z * lx), V(c2a1.x * ly, c2a1.y * ly, c2a1.z * ly));
            q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, ang2)));
        }
        q[JR_KROT] = kr;
        const M3 K = joint_mass_matrix(im1 + im2, U1, I1, U2, I2);
        M3 Kinv = m3_zero();
        const float det = m3_det(K);
        if (fabsf(det) > MACHINE_EPSILON) {
            if (dyn1 || dyn2) Kinv = m3_inverse(K, det);
            const v3 err = vsub(vsub(v3add(x2, r2), x1), r1);
            const v3 lam = m3_mulv(Kinv, vneg(err));
            x1 = v3add(x1, lin(im1, B1.lf, vneg(lam)));
            q1 = q_add_rot(q1, vcmul(B1.af, m3_mulv(I1, vcross(lam, r1))));
            x2 = v3add(x2, lin(im2, B2.lf, lam));
            q2 = q_add_rot(q2, vcmul(B2.af, m3_mulv(I2, vneg(vcross(lam, r2)))));
        }
        st3(q + JR_K, Kinv);
    }
    q[JR_STATE] = st;
    a.xc[e.y] = F4v(x1);
    a.xc[e.z] = F4v(x2);
    a.qc[e.y] = make_float4(q1.x, q1.y, q1.z, q1.w);
    a.qc[e.z] = make_float4(q2.x, q2.y, q2.z, q2.w);
}

}  // namespace rp3dg
