// Dynamics stage of a world step, after contact creation: world inverse
// inertia, velocity integration, the sequential-impulse contact solver with
// split impulses, position integration and the body / collider state update
// (reference src/engine/PhysicsWorld.cpp:239-318, src/systems/
// DynamicsSystem.cpp:44-183, src/systems/ContactSolverSystem.cpp:66-818).
//
// Five kernels: bodies (inertia + velocities), manifolds (solver records, one
// thread per manifold), islands (warm start, iterations, stored impulses: one
// thread per island, manifolds in the reference's order, so each island sees
// exactly the reference's sequence of Gauss-Seidel updates), bodies (positions
// + state), colliders (local-to-world).  Every expression keeps the
// reference's operand order; the library is built without FMA contraction,
// so results are bit-identical to the reference's float build.
#include <cuda_runtime.h>
#ifdef RP3DG_PROFILE_GIANT
#include <cstdio>
#endif

#include "broadphase_launch.h"
#include "dynamics_launch.h"
#include "rp3dg_math.cuh"

namespace rp3dg {

namespace {

constexpr float BETA = 0.2f;               // ContactSolverSystem.cpp:43
constexpr float BETA_SPLIT_IMPULSE = 0.2f;  // :44
constexpr float SLOP = 0.01f;              // :45

RD v3 L3(const float4 a) { return V(a.x, a.y, a.z); }
RD float4 F4(v3 a, float w = 0.0f) { return make_float4(a.x, a.y, a.z, w); }

// Matrix3x3 * Vector3 (Matrix3x3.h:324-331), row-major m[9]
RD v3 mv(const float* m, v3 v) {
    return V(m[0] * v.x + m[1] * v.y + m[2] * v.z,
             m[3] * v.x + m[4] * v.y + m[5] * v.z,
             m[6] * v.x + m[7] * v.y + m[8] * v.z);
}

// Quaternion::getMatrix (src/mathematics/Quaternion.cpp:138-165)
RD void quat_matrix(quat q, float* r) {
    const float nQ = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    float s = 0.0f;
    if (nQ > 0.0f) s = 2.0f / nQ;
    const float xs = q.x * s, ys = q.y * s, zs = q.z * s;
    const float wxs = q.w * xs, wys = q.w * ys, wzs = q.w * zs;
    const float xxs = q.x * xs, xys = q.x * ys, xzs = q.x * zs;
    const float yys = q.y * ys, yzs = q.y * zs, zzs = q.z * zs;
    r[0] = 1.0f - yys - zzs; r[1] = xys - wzs;        r[2] = xzs + wys;
    r[3] = xys + wzs;        r[4] = 1.0f - xxs - zzs; r[5] = yzs - wxs;
    r[6] = xzs - wys;        r[7] = yzs + wxs;        r[8] = 1.0f - xxs - yys;
}

// RigidBody::computeWorldInertiaTensorInverse (RigidBody.h:246-262):
// out = R * (diag(inv) * R^T), Matrix3x3 product of Matrix3x3.h:302-321
RD void world_inertia(const float* R, v3 inv, float* out) {
    float t[9];
    t[0] = R[0] * inv.x; t[1] = R[3] * inv.x; t[2] = R[6] * inv.x;
    t[3] = R[1] * inv.y; t[4] = R[4] * inv.y; t[5] = R[7] * inv.y;
    t[6] = R[2] * inv.z; t[7] = R[5] * inv.z; t[8] = R[8] * inv.z;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            out[3 * i + j] = R[3 * i + 0] * t[0 + j] + R[3 * i + 1] * t[3 + j] + R[3 * i + 2] * t[6 + j];
}

// v2 + w2 x r2 - v1 - w1 x r1, written out as in ContactSolverSystem.cpp:196-201
RD v3 rel_velocity(v3 v1, v3 w1, v3 v2, v3 w2, v3 r1, v3 r2) {
    return V(v2.x + w2.y * r2.z - w2.z * r2.y - v1.x - w1.y * r1.z + w1.z * r1.y,
             v2.y + w2.z * r2.x - w2.x * r2.z - v1.y - w1.z * r1.x + w1.x * r1.z,
             v2.z + w2.x * r2.y - w2.y * r2.x - v1.z - w1.x * r1.y + w1.y * r1.x);
}

// Vector3::getOneUnitOrthogonalVector (src/mathematics/Vector3.cpp:46-64)
RD v3 unit_orthogonal(v3 v) {
    const v3 a = V(fabsf(v.x), fabsf(v.y), fabsf(v.z));
    const int minElement = (a.x < a.y ? (a.x < a.z ? 0 : 2) : (a.y < a.z ? 1 : 2));
    if (minElement == 0) {
        const float l = sqrtf(v.y * v.y + v.z * v.z);
        return V(0.0f / l, -v.z / l, v.y / l);
    } else if (minElement == 1) {
        const float l = sqrtf(v.x * v.x + v.z * v.z);
        return V(-v.z / l, 0.0f / l, v.x / l);
    }
    const float l = sqrtf(v.x * v.x + v.y * v.y);
    return V(-v.y / l, v.x / l, 0.0f / l);
}

// Enabled bodies / colliders: the first nb_enabled / nc_enabled rows, or the
// rows flagged in b_enabled / c_enabled when those are given (several worlds
// in one batch, each with its own enabled range).
RD bool body_enabled(const DynArgs& a, uint32_t i) { return a.b_enabled ? a.b_enabled[i] != 0 : i < a.nb_enabled; }
RD bool collider_enabled(const DynArgs& a, uint32_t i) { return a.c_enabled ? a.c_enabled[i] != 0 : i < a.nc_enabled; }

// ---- kernel 1: world inverse inertia + velocity integration --------------
__global__ void __launch_bounds__(128) dyn_bodies_pre(const DynArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nb) return;
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    a.sv[i] = zero;
    a.sw[i] = zero;
    if (!body_enabled(a, i)) {
        // read-only body: the solver sees its stored velocity
        a.cv[i] = a.lin_vel[i];
        a.cw[i] = a.ang_vel[i];
        return;
    }
    // PhysicsWorld::updateBodiesInverseWorldInertiaTensors (:310-318)
    const float4 o = a.orientation[i];
    float R[9], I[9];
    quat_matrix(Q(o.x, o.y, o.z, o.w), R);
    world_inertia(R, L3(a.iil[i]), I);
    a.iiw[3 * i + 0] = make_float4(I[0], I[1], I[2], 0.0f);
    a.iiw[3 * i + 1] = make_float4(I[3], I[4], I[5], 0.0f);
    a.iiw[3 * i + 2] = make_float4(I[6], I[7], I[8], 0.0f);
    // DynamicsSystem::integrateRigidBodiesVelocities (DynamicsSystem.cpp:117-183)
    const float dt = a.dt;
    const float4 m = a.mass[i];  // mass, inverse mass, linear damping, angular damping
    const v3 lf = L3(a.llock[i]), af = L3(a.alock[i]);
    const v3 v = L3(a.lin_vel[i]), w = L3(a.ang_vel[i]);
    const v3 F = L3(a.force[i]);
    const float s = dt * m.y;
    v3 cv = V(v.x + s * lf.x * F.x, v.y + s * lf.y * F.y, v.z + s * lf.z * F.z);
    const v3 It = mv(I, L3(a.torque[i]));
    v3 cw = V(w.x + dt * af.x * It.x, w.y + dt * af.y * It.y, w.z + dt * af.z * It.z);
    if (a.gravity_enabled && a.gravity[i]) {
        cv = V(cv.x + s * lf.x * m.x * a.gx, cv.y + s * lf.y * m.x * a.gy, cv.z + s * lf.z * m.x * a.gz);
    }
    const float lin_damp = 1.0f / (1.0f + m.z * dt);
    const float ang_damp = 1.0f / (1.0f + m.w * dt);
    cv = vmul(cv, lin_damp);
    cw = vmul(cw, ang_damp);
    a.cv[i] = F4(cv);
    a.cw[i] = F4(cw);
}

RD bool is_fixed(const DynArgs& a, int32_t b) {
    if (uint32_t(b) >= a.nb || !body_enabled(a, uint32_t(b))) return true;
    const float4 il = a.iil[b];
    return a.mass[b].y == 0.0f && il.x == 0.0f && il.y == 0.0f && il.z == 0.0f;
}

RD float4 F4w(v3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// ---- kernel 2: ContactSolverSystem::initializeForIsland per manifold ------
// (ContactSolverSystem.cpp:116-318).  Writes the manifold's solver record and
// its points' records (layouts in dynamics_launch.h).
__global__ void __launch_bounds__(128) dyn_manifold_init(const DynArgs a) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.nm) return;
    float4* __restrict__ q = a.mrec[m].q;
    const int4 id = a.m_ids[m];
    const int32_t b1 = id.x, b2 = id.y;
    const uint32_t nb = a.m_npts[m], ps = a.m_pstart[m];
    if (uint32_t(b1) >= a.nb || uint32_t(b2) >= a.nb || b1 == b2 || uint32_t(id.z) >= a.nc ||
        uint32_t(id.w) >= a.nc || nb == 0 || nb > 4 || ps > a.np || nb > a.np - ps) {
        atomicOr(a.error, 4u);
        q[DQ_IDS] = make_float4(__int_as_float(0), __int_as_float(0), __int_as_float(0), __int_as_float(0));
        q[DQ_MASS] = make_float4(0.0f, 0.0f, 0.0f, 3.0f);  // no points: every pass skips it
        return;
    }
    q[DQ_IDS] = make_float4(__int_as_float(b1), __int_as_float(b2), __int_as_float(int32_t(nb)), __int_as_float(int32_t(ps)));
    const v3 x1 = L3(a.com_world[b1]), x2 = L3(a.com_world[b2]);
    float I1[9], I2[9];
    {
        const float4 r0 = a.iiw[3 * b1], r1 = a.iiw[3 * b1 + 1], r2 = a.iiw[3 * b1 + 2];
        I1[0] = r0.x; I1[1] = r0.y; I1[2] = r0.z; I1[3] = r1.x; I1[4] = r1.y; I1[5] = r1.z;
        I1[6] = r2.x; I1[7] = r2.y; I1[8] = r2.z;
        q[DQ_I1 + 0] = r0; q[DQ_I1 + 1] = r1; q[DQ_I1 + 2] = r2;
    }
    {
        const float4 r0 = a.iiw[3 * b2], r1 = a.iiw[3 * b2 + 1], r2 = a.iiw[3 * b2 + 2];
        I2[0] = r0.x; I2[1] = r0.y; I2[2] = r0.z; I2[3] = r1.x; I2[4] = r1.y; I2[5] = r1.z;
        I2[6] = r2.x; I2[7] = r2.y; I2[8] = r2.z;
        q[DQ_I2 + 0] = r0; q[DQ_I2 + 1] = r1; q[DQ_I2 + 2] = r2;
    }
    const float im1 = a.mass[b1].y, im2 = a.mass[b2].y;
    const float4 mat1 = a.c_mat[id.z], mat2 = a.c_mat[id.w];
    const float friction = mat1.x * mat2.x;                          // computeMixedFrictionCoefficient
    const float restitution = (mat1.y > mat2.y) ? mat1.y : mat2.y;   // computeMixedRestitutionFactor
    const float fixed = float((is_fixed(a, b1) ? 1 : 0) | (is_fixed(a, b2) ? 2 : 0));
    q[DQ_MASS] = make_float4(im1, im2, friction, fixed);
    q[DQ_LF1] = a.llock[b1]; q[DQ_LF2] = a.llock[b2];
    q[DQ_AF1] = a.alock[b1]; q[DQ_AF2] = a.alock[b2];
    const v3 v1 = L3(a.lin_vel[b1]), w1 = L3(a.ang_vel[b1]);
    const v3 v2 = L3(a.lin_vel[b2]), w2 = L3(a.ang_vel[b2]);
    const float4 o1 = a.c_wori[id.z], o2 = a.c_wori[id.w];
    const xform t1 = X(L3(a.c_wpos[id.z]), Q(o1.x, o1.y, o1.z, o1.w));
    const xform t2 = X(L3(a.c_wpos[id.w]), Q(o2.x, o2.y, o2.z, o2.w));
    v3 fp1 = V(0.0f, 0.0f, 0.0f), fp2 = V(0.0f, 0.0f, 0.0f), nsum = V(0.0f, 0.0f, 0.0f);
    for (uint32_t k = 0; k < nb; k++) {
        const uint32_t p = ps + k;
        DynPointRec& r = a.prec[p];
        const float4 nd = a.p_nd[p];
        const v3 n = V(nd.x, nd.y, nd.z);
        const v3 p1 = xapply(t1, L3(a.p_l1[p]));
        const v3 p2 = xapply(t2, L3(a.p_l2[p]));
        const v3 r1 = V(p1.x - x1.x, p1.y - x1.y, p1.z - x1.z);
        const v3 r2 = V(p2.x - x2.x, p2.y - x2.y, p2.z - x2.z);
        const uint8_t resting = a.p_resting[p];
        a.p_resting[p] = 1;
        fp1 = V(fp1.x + p1.x, fp1.y + p1.y, fp1.z + p1.z);
        fp2 = V(fp2.x + p2.x, fp2.y + p2.y, fp2.z + p2.z);
        const v3 dv = rel_velocity(v1, w1, v2, w2, r1, r2);
        const v3 r1n = vcross(r1, n), r2n = vcross(r2, n);
        const v3 i1 = mv(I1, r1n), i2 = mv(I2, r2n);
        const float mp = im1 + im2 + vdot(vcross(i1, r1), n) + vdot(vcross(i2, r2), n);
        const float inv_mass = mp > 0.0f ? 1.0f / mp : 0.0f;
        float bias = 0.0f;
        const float dvn = dv.x * n.x + dv.y * n.y + dv.z * n.z;
        if (dvn < -a.restitution_threshold) bias = restitution * dvn;
        r.q[DP_R1] = F4w(r1, nd.w);
        r.q[DP_R2] = F4w(r2, inv_mass);
        r.q[DP_N] = F4w(n, bias);
        r.q[DP_I1] = F4w(i1, 0.0f);
        r.q[DP_I2] = F4w(i2, 0.0f);
        r.mut = make_float4(a.p_impulse[p], 0.0f, resting ? 1.0f : 0.0f, 0.0f);
        nsum = V(nsum.x + n.x, nsum.y + n.y, nsum.z + n.z);
    }
    const float fnb = float(nb);
    fp1 = vdivs(fp1, fnb);
    fp2 = vdivs(fp2, fnb);
    const v3 r1f = V(fp1.x - x1.x, fp1.y - x1.y, fp1.z - x1.z);
    const v3 r2f = V(fp2.x - x2.x, fp2.y - x2.y, fp2.z - x2.z);
    q[DQ_OFV1] = a.m_fv1[m];
    q[DQ_OFV2] = a.m_fv2[m];
    const float4 fi = a.m_fimp[m];
    a.mrec[m].mut = make_float4(fi.x, fi.y, fi.z, 0.0f);
    const v3 n = vnormalize(nsum);
    // computeFrictionVectors (:789-818)
    const v3 dvf = rel_velocity(v1, w1, v2, w2, r1f, r2f);
    const float dvfn = vdot(dvf, n);
    const v3 nv = vmul(n, dvfn);
    const v3 tv = V(dvf.x - nv.x, dvf.y - nv.y, dvf.z - nv.z);
    const float lt = vlen(tv);
    const v3 fv1 = lt > MACHINE_EPSILON ? vdivs(tv, lt) : unit_orthogonal(n);
    const v3 fv2 = vcross(n, fv1);
    const v3 r1ct1 = vcross(r1f, fv1), r1ct2 = vcross(r1f, fv2);
    const v3 r2ct1 = vcross(r2f, fv1), r2ct2 = vcross(r2f, fv2);
    const float f1m = im1 + im2 + vdot(vcross(mv(I1, r1ct1), r1f), fv1) + vdot(vcross(mv(I2, r2ct1), r2f), fv1);
    const float f2m = im1 + im2 + vdot(vcross(mv(I1, r1ct2), r1f), fv2) + vdot(vcross(mv(I2, r2ct2), r2f), fv2);
    const float twm = vdot(n, mv(I1, n)) + vdot(n, mv(I2, n));
    q[DQ_N] = F4w(n, twm > 0.0f ? 1.0f / twm : 0.0f);
    q[DQ_R1F] = F4w(r1f, f1m > 0.0f ? 1.0f / f1m : 0.0f);
    q[DQ_R2F] = F4w(r2f, f2m > 0.0f ? 1.0f / f2m : 0.0f);
    q[DQ_FV1] = F4w(fv1, 0.0f);
    q[DQ_FV2] = F4w(fv2, 0.0f);
    q[DQ_R1CT1] = F4w(r1ct1, 0.0f);
    q[DQ_R1CT2] = F4w(r1ct2, 0.0f);
    q[DQ_R2CT1] = F4w(r2ct1, 0.0f);
    q[DQ_R2CT2] = F4w(r2ct2, 0.0f);
}

// A manifold's constant solver data in registers (one 16-byte load per row).
struct Man {
    int32_t b1, b2, nb, pstart;
    float im1, im2, friction;
    uint32_t fixed;
    v3 lf1, lf2, af1, af2;
    float I1[9], I2[9];
    v3 n, r1f, r2f, fv1, fv2, r1ct1, r1ct2, r2ct1, r2ct2;
    float inv_tw, inv_f1, inv_f2;
};

template <bool LDG>
RD float4 ldq(const float4* p) { return LDG ? __ldg(p) : *p; }

template <bool LDG>
RD void rows3(const float4* __restrict__ q, float* I) {
    const float4 r0 = ldq<LDG>(q), r1 = ldq<LDG>(q + 1), r2 = ldq<LDG>(q + 2);
    I[0] = r0.x; I[1] = r0.y; I[2] = r0.z; I[3] = r1.x; I[4] = r1.y; I[5] = r1.z;
    I[6] = r2.x; I[7] = r2.y; I[8] = r2.z;
}

// The records are written by kernel 2 and only read here, so the read-only
// data path may serve them (LDG); the giant-island kernel reads copies staged
// in shared memory (generic loads).
template <bool LDG = true>
RD void load_man_q(const float4* __restrict__ q, Man& c) {
    const float4 ids = ldq<LDG>(q + DQ_IDS), ms = ldq<LDG>(q + DQ_MASS);
    c.b1 = __float_as_int(ids.x); c.b2 = __float_as_int(ids.y);
    c.nb = __float_as_int(ids.z); c.pstart = __float_as_int(ids.w);
    c.im1 = ms.x; c.im2 = ms.y; c.friction = ms.z; c.fixed = uint32_t(ms.w);
    c.lf1 = L3(ldq<LDG>(q + DQ_LF1)); c.lf2 = L3(ldq<LDG>(q + DQ_LF2));
    c.af1 = L3(ldq<LDG>(q + DQ_AF1)); c.af2 = L3(ldq<LDG>(q + DQ_AF2));
    rows3<LDG>(q + DQ_I1, c.I1);
    rows3<LDG>(q + DQ_I2, c.I2);
    const float4 n = ldq<LDG>(q + DQ_N), r1f = ldq<LDG>(q + DQ_R1F), r2f = ldq<LDG>(q + DQ_R2F);
    c.n = L3(n); c.inv_tw = n.w;
    c.r1f = L3(r1f); c.inv_f1 = r1f.w;
    c.r2f = L3(r2f); c.inv_f2 = r2f.w;
    c.fv1 = L3(ldq<LDG>(q + DQ_FV1)); c.fv2 = L3(ldq<LDG>(q + DQ_FV2));
    c.r1ct1 = L3(ldq<LDG>(q + DQ_R1CT1)); c.r1ct2 = L3(ldq<LDG>(q + DQ_R1CT2));
    c.r2ct1 = L3(ldq<LDG>(q + DQ_R2CT1)); c.r2ct2 = L3(ldq<LDG>(q + DQ_R2CT2));
}
RD void load_man(const DynManifoldRec* __restrict__ rec, Man& c) { load_man_q<true>(rec->q, c); }

struct Pt {
    v3 r1, r2, n, i1, i2;
    float depth, inv_mass, bias;
};

template <bool LDG = true>
RD void load_pt_q(const float4* __restrict__ q, Pt& p) {
    const float4 a = ldq<LDG>(q + DP_R1), b = ldq<LDG>(q + DP_R2), c = ldq<LDG>(q + DP_N);
    p.r1 = L3(a); p.depth = a.w;
    p.r2 = L3(b); p.inv_mass = b.w;
    p.n = L3(c); p.bias = c.w;
    p.i1 = L3(ldq<LDG>(q + DP_I1));
    p.i2 = L3(ldq<LDG>(q + DP_I2));
}

// v -= im * imp * lock  /  v += im * imp * lock, per component (Vector3 operators)
RD v3 lin_sub(v3 v, float im, v3 imp, v3 lf) {
    return V(v.x - im * imp.x * lf.x, v.y - im * imp.y * lf.y, v.z - im * imp.z * lf.z);
}
RD v3 lin_add(v3 v, float im, v3 imp, v3 lf) {
    return V(v.x + im * imp.x * lf.x, v.y + im * imp.y * lf.y, v.z + im * imp.z * lf.z);
}
// w -= i * af * s  /  w += i * af * s, per component (the point updates)
RD v3 ang_sub(v3 w, v3 i, v3 af, float s) {
    return V(w.x - i.x * af.x * s, w.y - i.y * af.y * s, w.z - i.z * af.z * s);
}
RD v3 ang_add(v3 w, v3 i, v3 af, float s) {
    return V(w.x + i.x * af.x * s, w.y + i.y * af.y * s, w.z + i.z * af.z * s);
}

// Where the solver reads and writes the velocities (constrained and split)
// of a manifold's two bodies: the global scratch arrays, or a warp's shared
// memory copy for the movable bodies of a large island.
struct BodyVel {
    float4 *v1, *w1, *s1, *t1, *v2, *w2, *s2, *t2;
};

// Where the solver reads a manifold's constant rows and reads / writes its
// impulses: the records in global memory, or copies in shared memory.
// Point k's rows are at pq + k * pq_stride, its impulses at pmut + k * pmut_stride.
struct RecSrc {
    const float4* mq;
    float4* mmut;
    const float4* pq;
    float4* pmut;
    int pq_stride, pmut_stride;
};
constexpr int PREC_F4 = int(sizeof(DynPointRec) / sizeof(float4));
RD RecSrc rec_global(const DynArgs& a, uint32_t mi, int32_t pstart) {
    RecSrc r;
    r.mq = a.mrec[mi].q;
    r.mmut = &a.mrec[mi].mut;
    r.pq = a.prec[pstart].q;
    r.pmut = &a.prec[pstart].mut;
    r.pq_stride = PREC_F4;
    r.pmut_stride = PREC_F4;
    return r;
}

RD BodyVel vel_global(const DynArgs& a, int32_t b1, int32_t b2) {
    BodyVel p;
    p.v1 = a.cv + b1; p.w1 = a.cw + b1; p.s1 = a.sv + b1; p.t1 = a.sw + b1;
    p.v2 = a.cv + b2; p.w2 = a.cw + b2; p.s2 = a.sv + b2; p.t2 = a.sw + b2;
    return p;
}

// warmStart (:324-476) of one manifold: its two bodies' velocities are loaded,
// updated in the reference's statement order and stored back (the two bodies
// are distinct; fixed bodies are never stored).
// A manifold's point impulses held in four registers (PRE cores): loaded
// together before the points are solved and stored after, so that copies in
// global memory cost one round trip; points beyond four (none after the
// manifold step) are read and written in place.
RD void pmv_load(const RecSrc& r, int nb, float4& p0, float4& p1, float4& p2, float4& p3) {
    if (nb > 0) p0 = r.pmut[0];
    if (nb > 1) p1 = r.pmut[r.pmut_stride];
    if (nb > 2) p2 = r.pmut[2 * r.pmut_stride];
    if (nb > 3) p3 = r.pmut[3 * r.pmut_stride];
}
RD void pmv_store(const RecSrc& r, int nb, const float4& p0, const float4& p1, const float4& p2, const float4& p3) {
    if (nb > 0) r.pmut[0] = p0;
    if (nb > 1) r.pmut[r.pmut_stride] = p1;
    if (nb > 2) r.pmut[2 * r.pmut_stride] = p2;
    if (nb > 3) r.pmut[3 * r.pmut_stride] = p3;
}
template <bool PRE>
RD float4 pm_get(const RecSrc& r, int k, const float4& p0, const float4& p1, const float4& p2, const float4& p3) {
    if (!PRE) return r.pmut[k * r.pmut_stride];
    return k == 0 ? p0 : k == 1 ? p1 : k == 2 ? p2 : k == 3 ? p3 : r.pmut[k * r.pmut_stride];
}
template <bool PRE>
RD void pm_set(const RecSrc& r, int k, const float4& v, float4& p0, float4& p1, float4& p2, float4& p3) {
    if (!PRE || k > 3) { r.pmut[k * r.pmut_stride] = v; return; }
    if (k == 0) p0 = v;
    else if (k == 1) p1 = v;
    else if (k == 2) p2 = v;
    else p3 = v;
}

template <bool LDG, bool PRE = false>
RD void warm_core(const DynArgs& a, const RecSrc& r, const BodyVel& bv, int32_t nb) {
    if (nb == 0) return;  // rejected by the manifold kernel
    Man c;
    load_man_q<LDG>(r.mq, c);
    const v3 o1 = L3(ldq<LDG>(r.mq + DQ_OFV1)), o2 = L3(ldq<LDG>(r.mq + DQ_OFV2));
    float4 mut = *r.mmut;
    v3 v1 = L3(*bv.v1), w1 = L3(*bv.w1), v2 = L3(*bv.v2), w2 = L3(*bv.w2);
    float4 pv0, pv1, pv2, pv3;
    if (PRE) pmv_load(r, nb, pv0, pv1, pv2, pv3);
    bool resting_any = false;
    for (int k = 0; k < nb; k++) {
        float4 pm = pm_get<PRE>(r, k, pv0, pv1, pv2, pv3);
        if (pm.z != 0.0f) {
            resting_any = true;
            Pt p;
            load_pt_q<LDG>(r.pq + k * r.pq_stride, p);
            const float pi = pm.x;
            const v3 ip = V(p.n.x * pi, p.n.y * pi, p.n.z * pi);
            v1 = lin_sub(v1, c.im1, ip, c.lf1);
            w1 = ang_sub(w1, p.i1, c.af1, pi);
            v2 = lin_add(v2, c.im2, ip, c.lf2);
            w2 = ang_add(w2, p.i2, c.af2, pi);
        } else {
            pm.x = 0.0f;
            pm_set<PRE>(r, k, pm, pv0, pv1, pv2, pv3);
        }
    }
    if (PRE) pmv_store(r, nb, pv0, pv1, pv2, pv3);
    float f1 = mut.x, f2 = mut.y, ftw = mut.z;
    if (resting_any) {
        const v3 ofi = V(f1 * o1.x + f2 * o2.x, f1 * o1.y + f2 * o2.y, f1 * o1.z + f2 * o2.z);
        f1 = vdot(ofi, c.fv1);
        f2 = vdot(ofi, c.fv2);
        // first friction constraint
        v3 ai1 = V(-c.r1ct1.x * f1, -c.r1ct1.y * f1, -c.r1ct1.z * f1);
        v3 li2 = V(c.fv1.x * f1, c.fv1.y * f1, c.fv1.z * f1);
        v3 ai2 = V(c.r2ct1.x * f1, c.r2ct1.y * f1, c.r2ct1.z * f1);
        v1 = lin_sub(v1, c.im1, li2, c.lf1);
        w1 = vadd(w1, vcmul(c.af1, mv(c.I1, ai1)));
        v2 = lin_add(v2, c.im2, li2, c.lf2);
        w2 = vadd(w2, vcmul(c.af2, mv(c.I2, ai2)));
        // second friction constraint
        ai1 = V(-c.r1ct2.x * f2, -c.r1ct2.y * f2, -c.r1ct2.z * f2);
        li2 = V(c.fv2.x * f2, c.fv2.y * f2, c.fv2.z * f2);
        ai2 = V(c.r2ct2.x * f2, c.r2ct2.y * f2, c.r2ct2.z * f2);
        v1 = lin_sub(v1, c.im1, li2, c.lf1);
        w1 = vadd(w1, vcmul(c.af1, mv(c.I1, ai1)));
        v2 = lin_add(v2, c.im2, li2, c.lf2);
        w2 = vadd(w2, vcmul(c.af2, mv(c.I2, ai2)));
        // twist friction constraint (the reference applies the body-2
        // angular impulse to both bodies a second time, :461-465)
        ai1 = V(-c.n.x * ftw, -c.n.y * ftw, -c.n.z * ftw);
        ai2 = V(c.n.x * ftw, c.n.y * ftw, c.n.z * ftw);
        w1 = vadd(w1, vcmul(c.af1, mv(c.I1, ai1)));
        w2 = vadd(w2, vcmul(c.af2, mv(c.I2, ai2)));
        w1 = vsub(w1, vcmul(c.af1, mv(c.I1, ai2)));
        w2 = vadd(w2, vcmul(c.af2, mv(c.I2, ai2)));
    } else {
        f1 = 0.0f; f2 = 0.0f; ftw = 0.0f;
    }
    *r.mmut = make_float4(f1, f2, ftw, mut.w);
    if (!(c.fixed & 1)) { *bv.v1 = F4(v1); *bv.w1 = F4(w1); }
    if (!(c.fixed & 2)) { *bv.v2 = F4(v2); *bv.w2 = F4(w2); }
}
RD void warm_manifold(const DynArgs& a, uint32_t mi, const BodyVel& bv, int32_t nb, int32_t pstart) {
    warm_core<true>(a, rec_global(a, mi, pstart), bv, nb);
}

// One solve pass (:479-759) over one manifold.
template <bool LDG, bool PRE = false>
RD void solve_core(const DynArgs& a, const RecSrc& r, float beta, const BodyVel& bv, int32_t nb) {
    if (nb == 0) return;
    Man c;
    load_man_q<LDG>(r.mq, c);
    float4 mut = *r.mmut;
    v3 v1 = L3(*bv.v1), w1 = L3(*bv.w1), v2 = L3(*bv.v2), w2 = L3(*bv.w2);
    v3 s1 = L3(*bv.s1), t1 = L3(*bv.t1), s2 = L3(*bv.s2), t2 = L3(*bv.t2);
    float4 pv0, pv1, pv2, pv3;
    if (PRE) pmv_load(r, nb, pv0, pv1, pv2, pv3);
    float sum_pen = 0.0f;
    for (int k = 0; k < nb; k++) {
        Pt p;
        load_pt_q<LDG>(r.pq + k * r.pq_stride, p);
        float4 pm = pm_get<PRE>(r, k, pv0, pv1, pv2, pv3);
        const v3 n = p.n;
        const v3 dv = rel_velocity(v1, w1, v2, w2, p.r1, p.r2);
        const float Jv = dv.x * n.x + dv.y * n.y + dv.z * n.z;
        float bias_pen = 0.0f;
        if (p.depth > SLOP) {
            const float excess = p.depth - SLOP;
            bias_pen = -(beta / a.dt) * ((0.0f < excess) ? excess : 0.0f);
        }
        const float b = bias_pen + p.bias;
        float dl = a.split ? -(Jv + p.bias) * p.inv_mass : -(Jv + b) * p.inv_mass;
        const float lt = pm.x;
        const float sum = pm.x + dl;
        pm.x = (sum < 0.0f) ? 0.0f : sum;
        dl = pm.x - lt;
        const v3 li = V(n.x * dl, n.y * dl, n.z * dl);
        v1 = lin_sub(v1, c.im1, li, c.lf1);
        w1 = ang_sub(w1, p.i1, c.af1, dl);
        v2 = lin_add(v2, c.im2, li, c.lf2);
        w2 = ang_add(w2, p.i2, c.af2, dl);
        sum_pen += pm.x;
        if (a.split) {
            const v3 dvs = rel_velocity(s1, t1, s2, t2, p.r1, p.r2);
            const float Jvs = dvs.x * n.x + dvs.y * n.y + dvs.z * n.z;
            float dls = -(Jvs + bias_pen) * p.inv_mass;
            const float lts = pm.y;
            const float ss = pm.y + dls;
            pm.y = (ss < 0.0f) ? 0.0f : ss;
            dls = pm.y - lts;
            const v3 lis = V(n.x * dls, n.y * dls, n.z * dls);
            s1 = lin_sub(s1, c.im1, lis, c.lf1);
            t1 = ang_sub(t1, p.i1, c.af1, dls);
            s2 = lin_add(s2, c.im2, lis, c.lf2);
            t2 = ang_add(t2, p.i2, c.af2, dls);
        }
        pm_set<PRE>(r, k, pm, pv0, pv1, pv2, pv3);
    }
    if (PRE) pmv_store(r, nb, pv0, pv1, pv2, pv3);
    float f1 = mut.x, f2 = mut.y, ftw = mut.z;
    // first friction constraint
    {
        const v3 dv = rel_velocity(v1, w1, v2, w2, c.r1f, c.r2f);
        const float Jv = dv.x * c.fv1.x + dv.y * c.fv1.y + dv.z * c.fv1.z;
        float dl = -Jv * c.inv_f1;
        const float limit = c.friction * sum_pen;
        const float lt = f1;
        f1 = smax(-limit, smin(f1 + dl, limit));
        dl = f1 - lt;
        const v3 ai1 = V(-c.r1ct1.x * dl, -c.r1ct1.y * dl, -c.r1ct1.z * dl);
        const v3 li2 = V(c.fv1.x * dl, c.fv1.y * dl, c.fv1.z * dl);
        const v3 ai2 = V(c.r2ct1.x * dl, c.r2ct1.y * dl, c.r2ct1.z * dl);
        v1 = lin_sub(v1, c.im1, li2, c.lf1);
        w1 = vadd(w1, vcmul(c.af1, mv(c.I1, ai1)));
        v2 = lin_add(v2, c.im2, li2, c.lf2);
        w2 = vadd(w2, vcmul(c.af2, mv(c.I2, ai2)));
    }
    // second friction constraint
    {
        const v3 dv = rel_velocity(v1, w1, v2, w2, c.r1f, c.r2f);
        const float Jv = dv.x * c.fv2.x + dv.y * c.fv2.y + dv.z * c.fv2.z;
        float dl = -Jv * c.inv_f2;
        const float limit = c.friction * sum_pen;
        const float lt = f2;
        f2 = smax(-limit, smin(f2 + dl, limit));
        dl = f2 - lt;
        const v3 ai1 = V(-c.r1ct2.x * dl, -c.r1ct2.y * dl, -c.r1ct2.z * dl);
        const v3 li2 = V(c.fv2.x * dl, c.fv2.y * dl, c.fv2.z * dl);
        const v3 ai2 = V(c.r2ct2.x * dl, c.r2ct2.y * dl, c.r2ct2.z * dl);
        v1 = lin_sub(v1, c.im1, li2, c.lf1);
        w1 = vadd(w1, vcmul(c.af1, mv(c.I1, ai1)));
        v2 = lin_add(v2, c.im2, li2, c.lf2);
        w2 = vadd(w2, vcmul(c.af2, mv(c.I2, ai2)));
    }
    // twist friction constraint
    {
        const v3 dw = vsub(w2, w1);
        const float Jv = dw.x * c.n.x + dw.y * c.n.y + dw.z * c.n.z;
        float dl = -Jv * c.inv_tw;
        const float limit = c.friction * sum_pen;
        const float lt = ftw;
        ftw = smax(-limit, smin(ftw + dl, limit));
        dl = ftw - lt;
        const v3 ai2 = V(c.n.x * dl, c.n.y * dl, c.n.z * dl);
        w1 = vsub(w1, vcmul(c.af1, mv(c.I1, ai2)));
        w2 = vadd(w2, vcmul(c.af2, mv(c.I2, ai2)));
    }
    *r.mmut = make_float4(f1, f2, ftw, mut.w);
    if (!(c.fixed & 1)) { *bv.v1 = F4(v1); *bv.w1 = F4(w1); *bv.s1 = F4(s1); *bv.t1 = F4(t1); }
    if (!(c.fixed & 2)) { *bv.v2 = F4(v2); *bv.w2 = F4(w2); *bv.s2 = F4(s2); *bv.t2 = F4(t2); }
}
RD void solve_manifold(const DynArgs& a, uint32_t mi, float beta, const BodyVel& bv, int32_t nb, int32_t pstart) {
    solve_core<true>(a, rec_global(a, mi, pstart), beta, bv, nb);
}

// storeImpulses (:763-785) of one manifold.
RD void store_manifold(const DynArgs& a, uint32_t mi) {
    Man c;
    load_man(a.mrec + mi, c);
    if (c.nb == 0) return;
    for (int k = 0; k < c.nb; k++) a.p_impulse[c.pstart + k] = a.prec[c.pstart + k].mut.x;
    const float4 mut = a.mrec[mi].mut;
    a.m_fimp[mi] = make_float4(mut.x, mut.y, mut.z, 0.0f);
    a.m_fv1[mi] = F4(c.fv1);
    a.m_fv2[mi] = F4(c.fv2);
}

// ---- kernel 3: warm start, velocity iterations, stored impulses ----------
//
// The reference runs the manifolds of an island strictly in order; manifold j
// only reads and writes the velocities of its two bodies, and islands share
// only fixed bodies (static or kinematic: never written here).  So islands
// are independent, and inside an island any schedule that keeps, for every
// movable body, the order of the manifolds touching it gives bit-identical
// results.
//
// 3a: one thread per island runs islands of up to small_max manifolds in
//     the reference's order and queues the larger ones.
// 3b: persistent warps take the queued islands.  Lane 0 gives each manifold a
//     level (1 + the highest level of an earlier manifold sharing a movable
//     body) and sorts the island's manifolds by level; every pass (warm
//     start, each velocity iteration) then runs level after level, the
//     manifolds of a level in parallel across the warp, __syncwarp (which
//     orders the lanes' memory accesses) between levels.  An island of up to
//     STAGE_MANIFOLDS manifolds and STAGE_BODIES movable bodies is staged in
//     the warp's shared memory: its manifold table, the schedule (computed
//     with a shared hash of body -> slot, last level) and the bodies'
//     velocities.  Larger islands use the same schedule built in global
//     scratch, with velocities in global memory.

// (a.small_max, 8 by default, and a.giant_min, 256 by default: islands above
// it go to kernel 3c, one CTA per island, the island staged in up to the
// whole opt-in shared memory of a CTA; both come from DynTuning)
constexpr uint32_t BIG_ISLAND = 64;   // queued first: the longest islands start first

RD int4 man_ids(const DynArgs& a, uint32_t mi) {
    const float4 q = __ldg(a.mrec[mi].q + DQ_IDS);
    return make_int4(__float_as_int(q.x), __float_as_int(q.y), __float_as_int(q.z), __float_as_int(q.w));
}
RD uint32_t man_fixed(const DynArgs& a, uint32_t mi) { return uint32_t(__ldg(a.mrec[mi].q + DQ_MASS).w); }

__global__ void __launch_bounds__(128) dyn_islands_small(const DynArgs a) {
    const uint32_t is = blockIdx.x * blockDim.x + threadIdx.x;
    if (is >= a.ni) return;
    const uint32_t m0 = a.i_start[is], cnt = a.i_count[is];
    if (m0 > a.nm || cnt > a.nm - m0) {
        atomicOr(a.error, 4u);
        return;
    }
    if (a.i_jcount && a.i_jcount[is]) return;  // kernel 3d
    if (cnt == 0) return;
    if (cnt > a.small_max) {
        // big islands fill the list from the front, the others from the back
        if (cnt > a.giant_min) a.giant_list[atomicAdd(a.counters + 3, 1u)] = is;
        else if (cnt > BIG_ISLAND) a.large_list[atomicAdd(a.counters, 1u)] = is;
        else a.large_list[a.ni - 1 - atomicAdd(a.counters + 2, 1u)] = is;
        return;
    }
    const uint32_t m1 = m0 + cnt;
    for (uint32_t mi = m0; mi < m1; mi++) {
        const int4 id = man_ids(a, mi);
        warm_manifold(a, mi, vel_global(a, id.x, id.y), id.z, id.w);
    }
    const float beta = a.split ? BETA_SPLIT_IMPULSE : BETA;
    for (int it = 0; it < a.iterations; it++)
        for (uint32_t mi = m0; mi < m1; mi++) {
            const int4 id = man_ids(a, mi);
            solve_manifold(a, mi, beta, vel_global(a, id.x, id.y), id.z, id.w);
        }
    for (uint32_t mi = m0; mi < m1; mi++) store_manifold(a, mi);
}

// Shared memory of one warp of kernel 3b.
constexpr uint32_t STAGE_HASH = 2 * STAGE_BODIES;   // open addressing, load <= 1/2
struct WarpStage {
    float4 vel[4][STAGE_BODIES];        // constrained v, w and split v, w of the staged bodies
    int4 man[STAGE_MANIFOLDS];          // body 1, body 2, points, first point
    short2 slot[STAGE_MANIFOLDS];       // slot of body 1 / body 2 (-1: fixed body)
    uint16_t order[STAGE_MANIFOLDS];    // island manifolds sorted by level
    uint16_t lev[STAGE_MANIFOLDS];      // start of each level
    uint16_t klev[STAGE_MANIFOLDS];     // level of each manifold
    int32_t hkey[STAGE_HASH];           // body id (-1 empty)
    uint32_t hval[STAGE_HASH];          // slot << 16 | last level
    int32_t slot_body[STAGE_BODIES];    // body of each slot
};
static_assert(sizeof(WarpStage) <= LARGE_WARP_SMEM, "warp stage");

// Slot and last level of a movable body (inserted on first use); false when
// the island has more movable bodies than the stage holds.
RD bool stage_body(WarpStage* st, int32_t b, uint32_t& nslots, uint32_t& idx) {
    uint32_t h = (uint32_t(b) * 2654435761u) >> 23;   // 9 bits: STAGE_HASH = 512
    for (uint32_t probe = 0; probe < STAGE_HASH; probe++, h = (h + 1) & (STAGE_HASH - 1)) {
        const int32_t k = st->hkey[h];
        if (k == b) { idx = h; return true; }
        if (k < 0) {
            if (nslots >= STAGE_BODIES) return false;
            st->hkey[h] = b;
            st->hval[h] = nslots << 16;
            st->slot_body[nslots] = b;
            nslots++;
            idx = h;
            return true;
        }
    }
    return false;
}

// Schedule of a staged island in shared memory; false if it does not fit.
RD bool schedule_staged(const DynArgs& a, uint32_t m0, uint32_t cnt, WarpStage* st, uint32_t lane,
                        uint32_t& depth, uint32_t& nslots) {
    for (uint32_t h = lane; h < STAGE_HASH; h += 32) st->hkey[h] = -1;
    for (uint32_t k = lane; k < cnt; k += 32) {
        int4 id = man_ids(a, m0 + k);
        const uint32_t fixed = man_fixed(a, m0 + k);
        // fixed bodies are marked by a negative id in the table
        if (fixed & 1) id.x = -1 - id.x;
        if (fixed & 2) id.y = -1 - id.y;
        st->man[k] = id;
    }
    __syncwarp();
    bool ok = true;
    if (lane == 0) {
        depth = 0;
        nslots = 0;
        for (uint32_t k = 0; k < cnt && ok; k++) {
            const int4 id = st->man[k];
            uint32_t L = 1;
            short2 sl = make_short2(-1, -1);
            if (id.z != 0) {
                uint32_t h1 = 0, h2 = 0, l1 = 0, l2 = 0;
                if (id.x >= 0) { ok = stage_body(st, id.x, nslots, h1); if (ok) { l1 = st->hval[h1] & 0xffffu; sl.x = short(st->hval[h1] >> 16); } }
                if (ok && id.y >= 0) { ok = stage_body(st, id.y, nslots, h2); if (ok) { l2 = st->hval[h2] & 0xffffu; sl.y = short(st->hval[h2] >> 16); } }
                if (!ok) break;
                L = 1 + (l1 > l2 ? l1 : l2);
                if (id.x >= 0) st->hval[h1] = (st->hval[h1] & 0xffff0000u) | L;
                if (id.y >= 0) st->hval[h2] = (st->hval[h2] & 0xffff0000u) | L;
            }
            st->slot[k] = sl;
            st->klev[k] = uint16_t(L);
            depth = L > depth ? L : depth;
        }
        if (ok) {
            for (uint32_t L = 0; L < depth; L++) st->lev[L] = 0;
            for (uint32_t k = 0; k < cnt; k++) st->lev[st->klev[k] - 1]++;
            uint32_t run = 0;
            for (uint32_t L = 0; L < depth; L++) { run += st->lev[L]; st->lev[L] = uint16_t(run); }
            for (uint32_t k = cnt; k-- > 0;) st->order[--st->lev[st->klev[k] - 1]] = uint16_t(k);
        }
    }
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    depth = __shfl_sync(0xffffffffu, depth, 0);
    nslots = __shfl_sync(0xffffffffu, nslots, 0);
    __syncwarp();
    return ok;
}

RD void solve_staged(const DynArgs& a, uint32_t m0, uint32_t cnt, WarpStage* st, uint32_t lane, uint32_t depth,
                     uint32_t nslots) {
    for (uint32_t s = lane; s < nslots; s += 32) {
        const int32_t b = st->slot_body[s];
        st->vel[0][s] = a.cv[b]; st->vel[1][s] = a.cw[b];
        st->vel[2][s] = a.sv[b]; st->vel[3][s] = a.sw[b];
    }
    __syncwarp();
    const float beta = a.split ? BETA_SPLIT_IMPULSE : BETA;
    for (int pass = 0; pass <= a.iterations; pass++) {
        for (uint32_t L = 0; L < depth; L++) {
            const uint32_t b = st->lev[L];
            const uint32_t e = (L + 1 < depth) ? st->lev[L + 1] : cnt;
            for (uint32_t k = b + lane; k < e; k += 32) {
                const uint32_t kk = st->order[k];
                const int4 id = st->man[kk];
                const short2 sl = st->slot[kk];
                BodyVel bv;
                if (sl.x >= 0) { bv.v1 = &st->vel[0][sl.x]; bv.w1 = &st->vel[1][sl.x]; bv.s1 = &st->vel[2][sl.x]; bv.t1 = &st->vel[3][sl.x]; }
                else { const int32_t b1 = -1 - id.x; bv.v1 = a.cv + b1; bv.w1 = a.cw + b1; bv.s1 = a.sv + b1; bv.t1 = a.sw + b1; }
                if (sl.y >= 0) { bv.v2 = &st->vel[0][sl.y]; bv.w2 = &st->vel[1][sl.y]; bv.s2 = &st->vel[2][sl.y]; bv.t2 = &st->vel[3][sl.y]; }
                else { const int32_t b2 = -1 - id.y; bv.v2 = a.cv + b2; bv.w2 = a.cw + b2; bv.s2 = a.sv + b2; bv.t2 = a.sw + b2; }
                if (pass == 0) warm_manifold(a, m0 + kk, bv, id.z, id.w);
                else solve_manifold(a, m0 + kk, beta, bv, id.z, id.w);
            }
            __syncwarp();
        }
    }
    for (uint32_t s = lane; s < nslots; s += 32) {
        const int32_t b = st->slot_body[s];
        a.cv[b] = st->vel[0][s]; a.cw[b] = st->vel[1][s];
        a.sv[b] = st->vel[2][s]; a.sw[b] = st->vel[3][s];
    }
}

// Islands too large for the stage: the same schedule in global scratch.
RD void solve_global(const DynArgs& a, uint32_t m0, uint32_t cnt, uint32_t lane) {
    uint32_t* __restrict__ ord = a.order + m0;
    uint32_t* __restrict__ lev = a.level + m0;
    uint32_t* __restrict__ blev = a.body_level;
    for (uint32_t k = lane; k < cnt; k += 32) {
        const int4 id = man_ids(a, m0 + k);
        if (id.z == 0) continue;
        const uint32_t fixed = man_fixed(a, m0 + k);
        if (!(fixed & 1)) blev[id.x] = 0;
        if (!(fixed & 2)) blev[id.y] = 0;
    }
    __syncwarp();
    uint32_t depth = 0;
    if (lane == 0) {
        for (uint32_t k = 0; k < cnt; k++) {
            const int4 id = man_ids(a, m0 + k);
            uint32_t L = 1;
            if (id.z != 0) {
                const uint32_t fixed = man_fixed(a, m0 + k);
                const uint32_t l1 = (fixed & 1) ? 0u : blev[id.x];
                const uint32_t l2 = (fixed & 2) ? 0u : blev[id.y];
                L = 1 + (l1 > l2 ? l1 : l2);
                if (!(fixed & 1)) blev[id.x] = L;
                if (!(fixed & 2)) blev[id.y] = L;
            }
            ord[k] = L;  // the level, until the scatter below
            depth = L > depth ? L : depth;
        }
        for (uint32_t L = 0; L < depth; L++) lev[L] = 0;
        for (uint32_t k = 0; k < cnt; k++) lev[ord[k] - 1]++;
        uint32_t run = 0;
        for (uint32_t L = 0; L < depth; L++) { run += lev[L]; lev[L] = run; }
        // keep the levels in the records' spare word while scattering
        for (uint32_t k = 0; k < cnt; k++) a.mrec[m0 + k].mut.w = __int_as_float(int32_t(ord[k]));
        for (uint32_t k = cnt; k-- > 0;) {
            const uint32_t L = uint32_t(__float_as_int(a.mrec[m0 + k].mut.w));
            ord[--lev[L - 1]] = k;
        }
    }
    depth = __shfl_sync(0xffffffffu, depth, 0);
    __syncwarp();
    const float beta = a.split ? BETA_SPLIT_IMPULSE : BETA;
    for (int pass = 0; pass <= a.iterations; pass++) {
        for (uint32_t L = 0; L < depth; L++) {
            const uint32_t b = lev[L];
            const uint32_t e = (L + 1 < depth) ? lev[L + 1] : cnt;
            for (uint32_t k = b + lane; k < e; k += 32) {
                const uint32_t mi = m0 + ord[k];
                const int4 id = man_ids(a, mi);
                if (pass == 0) warm_manifold(a, mi, vel_global(a, id.x, id.y), id.z, id.w);
                else solve_manifold(a, mi, beta, vel_global(a, id.x, id.y), id.z, id.w);
            }
            __syncwarp();
        }
    }
}

__global__ void __launch_bounds__(LARGE_WARPS * 32, 2) dyn_islands_large(const DynArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpStage* st = reinterpret_cast<WarpStage*>(smem_raw + size_t(wid) * LARGE_WARP_SMEM);
    const uint32_t n_big = a.counters[0], n_mid = a.counters[2];
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(a.counters + 1, 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= n_big + n_mid) break;
        const uint32_t is = k < n_big ? a.large_list[k] : a.large_list[a.ni - 1 - (k - n_big)];
        const uint32_t m0 = a.i_start[is], cnt = a.i_count[is];
        uint32_t depth = 0, nslots = 0;
        if (cnt <= STAGE_MANIFOLDS && schedule_staged(a, m0, cnt, st, lane, depth, nslots))
            solve_staged(a, m0, cnt, st, lane, depth, nslots);
        else
            solve_global(a, m0, cnt, lane);
        for (uint32_t j = lane; j < cnt; j += 32) store_manifold(a, m0 + j);
        __syncwarp();
    }
}


}  // namespace
}  // namespace rp3dg
#include "joints.cuh"
namespace rp3dg {
namespace {

// ---- kernel 3d: islands with joints --------------------------------------
//
// One thread per island, in the reference's order: the contact warm start
// (ContactSolverSystem::init), the joints' warm start
// (ConstraintSolverSystem::initialize: ball-and-socket, then hinge), then per
// velocity iteration the joints (solveVelocityConstraints) before the
// contacts (ContactSolverSystem::solve), and storeImpulses.
__global__ void __launch_bounds__(128) dyn_joints_init(const DynArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.nj) joint_init(a, a.j_list[i]);
}

__global__ void __launch_bounds__(64) dyn_islands_joint(const DynArgs a) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nji) return;
    const uint32_t is = a.ji_island[k];
    const uint32_t m0 = a.i_start[is], cnt = a.i_count[is];
    const uint32_t j0 = a.i_jstart[is], jn = a.i_jcount[is];
    if (m0 > a.nm || cnt > a.nm - m0 || j0 > a.nj || jn > a.nj - j0) {
        atomicOr(a.error, 4u);
        return;
    }
    for (uint32_t mi = m0; mi < m0 + cnt; mi++) {
        const int4 id = man_ids(a, mi);
        warm_manifold(a, mi, vel_global(a, id.x, id.y), id.z, id.w);
    }
    for (uint32_t j = j0; j < j0 + jn; j++) joint_warm(a, a.j_list[j]);
    const float beta = a.split ? BETA_SPLIT_IMPULSE : BETA;
    for (int it = 0; it < a.iterations; it++) {
        for (uint32_t j = j0; j < j0 + jn; j++) joint_solve(a, a.j_list[j]);
        for (uint32_t mi = m0; mi < m0 + cnt; mi++) {
            const int4 id = man_ids(a, mi);
            solve_manifold(a, mi, beta, vel_global(a, id.x, id.y), id.z, id.w);
        }
    }
    for (uint32_t mi = m0; mi < m0 + cnt; mi++) store_manifold(a, mi);
}

// ---- kernel 4b: position correction of the joints (solvePositionCorrection,
// PhysicsWorld.cpp:348-360) and updateBodiesState (DynamicsSystem.cpp:74-110)
// of the islands with joints.
__global__ void __launch_bounds__(64) dyn_joints_position(const DynArgs a) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nji) return;
    const uint32_t is = a.ji_island[k];
    const uint32_t j0 = a.i_jstart[is], jn = a.i_jcount[is];
    if (j0 > a.nj || jn > a.nj - j0) return;
    for (int it = 0; it < a.position_iterations; it++)
        for (uint32_t j = j0; j < j0 + jn; j++) joint_position(a, a.j_list[j]);
    for (uint32_t r = a.ji_bstart[k]; r < a.ji_bstart[k] + a.ji_bcount[k]; r++) {
        const int32_t i = a.ji_rows[r];
        const v3 cp = L3(a.xc[i]);
        const float4 c4 = a.qc[i];
        const quat co = Q(c4.x, c4.y, c4.z, c4.w);
        a.com_world[i] = F4(cp);
        const float len = sqrtf(co.x * co.x + co.y * co.y + co.z * co.z + co.w * co.w);
        const quat u = Q(co.x / len, co.y / len, co.z / len, co.w / len);
        a.orientation[i] = make_float4(u.x, u.y, u.z, u.w);
        const v3 rr = qrot(u, L3(a.com_local[i]));
        a.position[i] = F4(V(cp.x - rr.x, cp.y - rr.y, cp.z - rr.z));
    }
}

// ---- kernel 3c: islands of more than giant_min manifolds -----------------
//
// One CTA of two warps takes one island at a time with the CTA's whole opt-in
// shared memory: the movable bodies' velocities, every manifold's and point's
// impulses, the manifold table and the level schedule (built by lane 0 with a
// shared hash of body -> slot, last level) stay on chip for the warm start and
// all velocity iterations.  Warp 0 solves, level after level; warp 1 stages
// the constant rows of the manifolds (and their points) of level t + 2 into a
// three-level ring with cp.async, with a compact descriptor per manifold,
// while warp 0 solves level t, so warp 0's time per level is its arithmetic.
// The two warps meet at one named barrier per level.  The arithmetic is
// warm_core / solve_core, the same as the other paths: only where the rows and
// impulses live changes.  An island that does not fit falls back to the
// schedule in global scratch (solve_global), run by warp 0.
constexpr uint32_t GIANT_RING = 8;     // manifolds of a level staged (the first 8)
constexpr uint32_t GIANT_LEVELS = 3;   // levels in the ring
constexpr uint32_t GIANT_THREADS = 64;
struct __align__(16) GiantSlot {
    int4 desc;                         // slot 1 | slot 2 << 16 (0xffff: fixed), points, manifold (island index), first point
    float4 mq[DQ_ROWS];
    float4 pq[4 * PREC_F4];
};

RD void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
RD void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
RD void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
// named barrier 1 over both warps of the CTA
RD void giant_bar() { asm volatile("bar.sync 1, %0;\n" ::"n"(GIANT_THREADS) : "memory"); }

struct GiantStage {
    float4 *vel, *mmut, *pmut;
    GiantSlot* ring;
    int32_t *hkey, *slot_body;
    uint32_t* hval;
    int2* man;             // body ids (fixed bodies as -1 - id)
    short2* slot;          // staged slot of body 1 / body 2 (-1: fixed)
    uint16_t *order, *klev, *lev;
    uint32_t* pofs;        // first point of each manifold, relative to the island's first point
    uint8_t* npt;
    uint32_t H, nbmax;
};

RD bool giant_layout(const DynArgs& a, uint32_t cnt, uint32_t np, unsigned char* sm, GiantStage& g) {
    if (cnt > 65535u) return false;
    g.nbmax = 2 * cnt < a.nb ? 2 * cnt : a.nb;
    if (g.nbmax > 32767u) return false;
    g.H = 1;
    while (g.H < 2 * g.nbmax) g.H <<= 1;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off = (off + bytes + 15) & ~size_t(15); return sm + o; };
    g.vel = reinterpret_cast<float4*>(take(size_t(4) * g.nbmax * 16));
    g.mmut = reinterpret_cast<float4*>(take(size_t(cnt) * 16));
    g.pmut = reinterpret_cast<float4*>(take(size_t(np) * 16));
    g.ring = reinterpret_cast<GiantSlot*>(take(size_t(GIANT_LEVELS) * GIANT_RING * sizeof(GiantSlot)));
    g.hkey = reinterpret_cast<int32_t*>(take(size_t(g.H) * 4));
    g.hval = reinterpret_cast<uint32_t*>(take(size_t(g.H) * 4));
    g.slot_body = reinterpret_cast<int32_t*>(take(size_t(g.nbmax) * 4));
    g.man = reinterpret_cast<int2*>(take(size_t(cnt) * 8));
    g.slot = reinterpret_cast<short2*>(take(size_t(cnt) * 4));
    g.order = reinterpret_cast<uint16_t*>(take(size_t(cnt) * 2));
    g.klev = reinterpret_cast<uint16_t*>(take(size_t(cnt) * 2));
    g.lev = reinterpret_cast<uint16_t*>(take(size_t(cnt + 1) * 2));
    g.pofs = reinterpret_cast<uint32_t*>(take(size_t(cnt) * 4));
    g.npt = take(size_t(cnt));
    return off <= a.giant_smem;
}

RD bool giant_body(GiantStage& g, int32_t b, uint32_t& nslots, uint32_t& idx) {
    uint32_t h = (uint32_t(b) * 2654435761u) & (g.H - 1);
    for (uint32_t probe = 0; probe < g.H; probe++, h = (h + 1) & (g.H - 1)) {
        const int32_t k = g.hkey[h];
        if (k == b) { idx = h; return true; }
        if (k < 0) {
            if (nslots >= g.nbmax) return false;
            g.hkey[h] = b;
            g.hval[h] = nslots << 16;
            g.slot_body[nslots] = b;
            nslots++;
            idx = h;
            return true;
        }
    }
    return false;
}

// Stage and schedule an island (warp 0); false (nothing written to global
// memory) when it does not fit or its points are not one contiguous range.
RD bool giant_schedule(const DynArgs& a, uint32_t m0, uint32_t cnt, unsigned char* sm, GiantStage& g,
                       uint32_t lane, uint32_t& depth, uint32_t& nslots, uint32_t& p0) {
    const int4 f = man_ids(a, m0), l = man_ids(a, m0 + cnt - 1);
    p0 = uint32_t(f.w);
    const int64_t end = int64_t(l.w) + int64_t(l.z);
    if (f.w < 0 || end < int64_t(p0) || end > int64_t(a.np)) return false;
    const uint32_t np = uint32_t(end - int64_t(p0));
    if (!giant_layout(a, cnt, np, sm, g)) return false;
    for (uint32_t h = lane; h < g.H; h += 32) g.hkey[h] = -1;
    for (uint32_t k = lane; k < cnt; k += 32) {
        const int4 id = man_ids(a, m0 + k);
        const uint32_t fixed = man_fixed(a, m0 + k);
        g.man[k] = make_int2((fixed & 1) ? -1 - id.x : id.x, (fixed & 2) ? -1 - id.y : id.y);
        g.pofs[k] = uint32_t(id.w) - p0;
        g.npt[k] = uint8_t(id.z < 0 ? 0 : (id.z > 255 ? 255 : id.z));
    }
    __syncwarp();
    bool ok = true;
    if (lane == 0) {
        depth = 0;
        nslots = 0;
        uint32_t expect = 0;
        for (uint32_t k = 0; k < cnt && ok; k++) {
            const int2 id = g.man[k];
            if (g.pofs[k] != expect || g.npt[k] > 4) { ok = false; break; }
            expect += g.npt[k];
            uint32_t L = 1;
            short2 sl = make_short2(-1, -1);
            if (g.npt[k] != 0) {
                uint32_t h1 = 0, h2 = 0, l1 = 0, l2 = 0;
                if (id.x >= 0) { ok = giant_body(g, id.x, nslots, h1); if (ok) { l1 = g.hval[h1] & 0xffffu; sl.x = short(g.hval[h1] >> 16); } }
                if (ok && id.y >= 0) { ok = giant_body(g, id.y, nslots, h2); if (ok) { l2 = g.hval[h2] & 0xffffu; sl.y = short(g.hval[h2] >> 16); } }
                if (!ok) break;
                L = 1 + (l1 > l2 ? l1 : l2);
                if (id.x >= 0) g.hval[h1] = (g.hval[h1] & 0xffff0000u) | L;
                if (id.y >= 0) g.hval[h2] = (g.hval[h2] & 0xffff0000u) | L;
            }
            g.slot[k] = sl;
            g.klev[k] = uint16_t(L);
            depth = L > depth ? L : depth;
        }
        if (ok && expect != np) ok = false;
        if (ok) {
            for (uint32_t L = 0; L <= depth; L++) g.lev[L] = 0;
            for (uint32_t k = 0; k < cnt; k++) g.lev[g.klev[k] - 1]++;
            uint32_t run = 0;
            for (uint32_t L = 0; L < depth; L++) { run += g.lev[L]; g.lev[L] = uint16_t(run); }
            g.lev[depth] = uint16_t(cnt);
            for (uint32_t k = cnt; k-- > 0;) g.order[--g.lev[g.klev[k] - 1]] = uint16_t(k);
        }
    }
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    depth = __shfl_sync(0xffffffffu, depth, 0);
    nslots = __shfl_sync(0xffffffffu, nslots, 0);
    __syncwarp();
    return ok;
}

// Warp 1: stage level t (of the linearised passes x levels) into ring level t % 3.
RD void giant_stage_level(const DynArgs& a, const GiantStage& g, uint32_t m0, uint32_t p0, uint32_t depth,
                          uint32_t total, uint32_t t, uint32_t lane) {
    if (t < total) {
        const uint32_t L = t % depth;
        const uint32_t j = g.lev[L] + lane;
        if (lane < GIANT_RING && j < g.lev[L + 1]) {
            const uint32_t kk = g.order[j];
            GiantSlot* sl = g.ring + (t % GIANT_LEVELS) * GIANT_RING + lane;
            const short2 bs = g.slot[kk];
            const uint32_t np = g.npt[kk];
            sl->desc = make_int4(int(uint32_t(uint16_t(bs.x)) | (uint32_t(uint16_t(bs.y)) << 16)), int(np), int(kk),
                                 int(g.pofs[kk]));
            const float4* src = a.mrec[m0 + kk].q;
            for (int r = 0; r < DQ_ROWS; r++) cp_async16(&sl->mq[r], src + r);
            const float4* ps = a.prec[p0 + g.pofs[kk]].q;
            for (uint32_t r = 0; r < np * PREC_F4; r++) cp_async16(&sl->pq[r], ps + r);
        }
    }
    cp_async_commit();
}

RD BodyVel giant_vel(const DynArgs& a, const GiantStage& g, int32_t s1, int32_t s2, int2 id) {
    BodyVel bv;
    const uint32_t n = g.nbmax;
    if (s1 >= 0) { bv.v1 = g.vel + s1; bv.w1 = g.vel + n + s1; bv.s1 = g.vel + 2 * n + s1; bv.t1 = g.vel + 3 * n + s1; }
    else { const int32_t b1 = -1 - id.x; bv.v1 = a.cv + b1; bv.w1 = a.cw + b1; bv.s1 = a.sv + b1; bv.t1 = a.sw + b1; }
    if (s2 >= 0) { bv.v2 = g.vel + s2; bv.w2 = g.vel + n + s2; bv.s2 = g.vel + 2 * n + s2; bv.t2 = g.vel + 3 * n + s2; }
    else { const int32_t b2 = -1 - id.y; bv.v2 = a.cv + b2; bv.w2 = a.cw + b2; bv.s2 = a.sv + b2; bv.t2 = a.sw + b2; }
    return bv;
}

// Both warps: stage, solve and write back one island.
RD void giant_solve(const DynArgs& a, uint32_t m0, uint32_t cnt, const GiantStage& g, uint32_t warp,
                    uint32_t lane, uint32_t depth, uint32_t nslots, uint32_t p0) {
    const uint32_t np = g.pofs[cnt - 1] + g.npt[cnt - 1];
    const uint32_t tid = warp * 32 + lane;
    for (uint32_t s = tid; s < nslots; s += GIANT_THREADS) {
        const int32_t b = g.slot_body[s];
        g.vel[s] = a.cv[b];
        g.vel[g.nbmax + s] = a.cw[b];
        g.vel[2 * g.nbmax + s] = a.sv[b];
        g.vel[3 * g.nbmax + s] = a.sw[b];
    }
    for (uint32_t k = tid; k < cnt; k += GIANT_THREADS) g.mmut[k] = a.mrec[m0 + k].mut;
    for (uint32_t p = tid; p < np; p += GIANT_THREADS) g.pmut[p] = a.prec[p0 + p].mut;
    const uint32_t total = uint32_t(a.iterations + 1) * depth;
    if (warp == 1) {
        giant_stage_level(a, g, m0, p0, depth, total, 0, lane);
        giant_stage_level(a, g, m0, p0, depth, total, 1, lane);
        cp_async_wait<1>();
        giant_bar();                       // level 0 staged, stage loads done
        for (uint32_t t = 0; t < total; t++) {
            giant_stage_level(a, g, m0, p0, depth, total, t + 2, lane);
            cp_async_wait<1>();            // level t + 1 staged
            giant_bar();                   // end of level t
        }
        cp_async_wait<0>();
    } else {
        const float beta = a.split ? BETA_SPLIT_IMPULSE : BETA;
        giant_bar();
        for (uint32_t t = 0; t < total; t++) {
            const uint32_t L = t % depth;
            const bool warm = t < depth;
            const uint32_t b = g.lev[L], e = g.lev[L + 1];
            if (lane < GIANT_RING && b + lane < e) {
                const GiantSlot* sl = g.ring + (t % GIANT_LEVELS) * GIANT_RING + lane;
                const int4 d = sl->desc;
                const int32_t s1 = int32_t(int16_t(d.x & 0xffff)), s2 = int32_t(int16_t(uint32_t(d.x) >> 16));
                const BodyVel bv = giant_vel(a, g, s1, s2, g.man[d.z]);
                RecSrc r;
                r.mq = sl->mq;
                r.pq = sl->pq;
                r.pq_stride = PREC_F4;
                r.mmut = g.mmut + d.z;
                r.pmut = g.pmut + d.w;
                r.pmut_stride = 1;
                if (warm) warm_core<false>(a, r, bv, d.y);
                else solve_core<false>(a, r, beta, bv, d.y);
            }
            // manifolds of a level beyond the staged ones read their rows from global memory
            for (uint32_t j = b + GIANT_RING + lane; j < e; j += 32) {
                const uint32_t kk = g.order[j];
                const short2 sl = g.slot[kk];
                const BodyVel bv = giant_vel(a, g, sl.x, sl.y, g.man[kk]);
                RecSrc r;
                r.mq = a.mrec[m0 + kk].q;
                r.pq = a.prec[p0 + g.pofs[kk]].q;
                r.pq_stride = PREC_F4;
                r.mmut = g.mmut + kk;
                r.pmut = g.pmut + g.pofs[kk];
                r.pmut_stride = 1;
                if (warm) warm_core<true>(a, r, bv, g.npt[kk]);
                else solve_core<true>(a, r, beta, bv, g.npt[kk]);
            }
            __syncwarp();
            giant_bar();
        }
    }
    __syncthreads();
    for (uint32_t s = tid; s < nslots; s += GIANT_THREADS) {
        const int32_t b = g.slot_body[s];
        a.cv[b] = g.vel[s];
        a.cw[b] = g.vel[g.nbmax + s];
        a.sv[b] = g.vel[2 * g.nbmax + s];
        a.sw[b] = g.vel[3 * g.nbmax + s];
    }
    for (uint32_t k = tid; k < cnt; k += GIANT_THREADS) a.mrec[m0 + k].mut = g.mmut[k];
    for (uint32_t p = tid; p < np; p += GIANT_THREADS) a.prec[p0 + p].mut = g.pmut[p];
    __syncthreads();
}

// ---- islands too large for shared memory: streamed ---------------------
//
// The level schedule is built by warp 0 in global scratch, 32 manifolds at a
// time: the lanes load their manifolds' bodies and the bodies' last levels in
// parallel, then a 32-step shuffle scan settles the dependencies inside the
// chunk in manifold order (a manifold's level is one more than the latest
// level of its movable bodies, exactly as the sequential rule).  A stable
// counting sort by level follows (histogram, scan, scatter with per-level
// ranks from __match_any_sync).  The solve is the giant pipeline with the
// island state left in global memory: warp 1 stages the constant rows of up
// to 32 manifolds per level two levels ahead, warp 0 solves each level from
// the ring with the velocities and impulses read from and written to global
// memory; both warps meet at the named barrier once per level.
constexpr uint32_t STREAM_RING = 32;

// Warp 0: levels and the level-ordered manifolds of an island.  Writes
// a.order[m0 + i] (island-relative manifold indices in level order) and
// a.level[m0 + L] = end of level L in that order; returns the depth.
RD uint32_t stream_schedule(const DynArgs& a, uint32_t m0, uint32_t cnt, uint32_t lane) {
    uint32_t* __restrict__ ord = a.order + m0;
    uint32_t* __restrict__ lev = a.level + m0;
    uint32_t* __restrict__ blev = a.body_level;
    for (uint32_t k = lane; k < cnt; k += 32) {
        const int4 id = man_ids(a, m0 + k);
        if (id.z == 0) continue;
        const uint32_t fixed = man_fixed(a, m0 + k);
        if (!(fixed & 1)) blev[id.x] = 0;
        if (!(fixed & 2)) blev[id.y] = 0;
    }
    __syncwarp();
    uint32_t depth = 0;
    for (uint32_t base = 0; base < cnt; base += 32) {
        const uint32_t k = base + lane;
        int32_t b1 = -1, b2 = -1;
        if (k < cnt) {
            const int4 id = man_ids(a, m0 + k);
            if (id.z != 0) {
                const uint32_t fixed = man_fixed(a, m0 + k);
                b1 = (fixed & 1) ? -1 : id.x;
                b2 = (fixed & 2) ? -1 : id.y;
            }
        }
        uint32_t l1 = b1 >= 0 ? blev[b1] : 0u, l2 = b2 >= 0 ? blev[b2] : 0u, L = 1;
        bool last1 = true, last2 = true;
        for (uint32_t j = 0; j < 32; j++) {
            if (lane == j) L = 1 + (l1 > l2 ? l1 : l2);
            const uint32_t Lj = __shfl_sync(0xffffffffu, L, int(j));
            const int32_t c1 = __shfl_sync(0xffffffffu, b1, int(j)), c2 = __shfl_sync(0xffffffffu, b2, int(j));
            const bool m1 = b1 >= 0 && (b1 == c1 || b1 == c2), m2 = b2 >= 0 && (b2 == c1 || b2 == c2);
            if (lane > j) {
                if (m1) l1 = Lj;
                if (m2) l2 = Lj;
            } else if (lane < j) {
                if (m1) last1 = false;
                if (m2) last2 = false;
            }
        }
        if (k < cnt) {
            if (b1 >= 0 && last1) blev[b1] = L;
            if (b2 >= 0 && last2) blev[b2] = L;
            // the level, kept in the record's spare word until the scatter
            a.mrec[m0 + k].mut.w = __int_as_float(int32_t(L));
            depth = L > depth ? L : depth;
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) {
        const uint32_t d = __shfl_xor_sync(0xffffffffu, depth, o);
        depth = d > depth ? d : depth;
    }
    // counting sort by level, stable in manifold order
    for (uint32_t L = lane; L < depth; L += 32) lev[L] = 0;
    __syncwarp();
    for (uint32_t k = lane; k < cnt; k += 32)
        atomicAdd(lev + (uint32_t(__float_as_int(a.mrec[m0 + k].mut.w)) - 1), 1u);
    __syncwarp();
    uint32_t run = 0;
    for (uint32_t base = 0; base < depth; base += 32) {
        const uint32_t L = base + lane;
        const uint32_t v = L < depth ? lev[L] : 0u;
        uint32_t inc = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= uint32_t(o)) inc += t;
        }
        if (L < depth) lev[L] = run + inc - v;   // first position of level L
        run += __shfl_sync(0xffffffffu, inc, 31);
    }
    __syncwarp();
    const uint32_t lt = (1u << lane) - 1u;
    for (uint32_t base = 0; base < cnt; base += 32) {
        const uint32_t k = base + lane;
        const uint32_t L = k < cnt ? uint32_t(__float_as_int(a.mrec[m0 + k].mut.w)) : 0u;
        const uint32_t key = k < cnt ? L : (0x80000000u | lane);
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        const uint32_t pos = k < cnt ? lev[L - 1] + uint32_t(__popc(peers & lt)) : 0u;
        __syncwarp();
        if (k < cnt) {
            ord[pos] = k;
            // the lowest lane of a level advances its cursor past the chunk's peers
            if ((peers & lt) == 0) lev[L - 1] += uint32_t(__popc(peers));
        }
        __syncwarp();
    }
    // lev[L] is now the end of level L
    return depth;
}

// Warp 1's staging pipeline: for linearised level x (passes x levels) it
// loads the level's bounds three steps ahead, the lanes' manifold indices two
// steps ahead and their id rows one step ahead, and issues the cp.async
// copies of the rows at x, so that no stage waits on a load issued in the
// same step; the registers then shift by one level.
struct StreamPipe {
    int2 b0, b1, b2;   // bounds of levels x, x + 1, x + 2
    uint32_t k0, k1;   // the lane's manifold of levels x, x + 1 (~0u: none)
    int4 i0;           // the id row of k0
};
RD int2 stream_bounds(const DynArgs& a, uint32_t m0, uint32_t depth, int64_t total, int64_t x) {
    if (x < 0 || x >= total) return make_int2(0, 0);
    const uint32_t L = uint32_t(x) % depth;
    return make_int2(int(L ? a.level[m0 + L - 1] : 0u), int(a.level[m0 + L]));
}
RD uint32_t stream_kk(const DynArgs& a, uint32_t m0, int2 bd, uint32_t lane) {
    const uint32_t j = uint32_t(bd.x) + lane;
    return (lane < STREAM_RING && j < uint32_t(bd.y)) ? a.order[m0 + j] : ~0u;
}

// One pipeline step for level x (negative in the prologue: loads only); the
// header of level x (its bounds) goes to hdr[x % 3] for warp 0.
RD void stream_stage_step(const DynArgs& a, GiantSlot* ring, int2* hdr, StreamPipe& P, uint32_t m0, uint32_t depth,
                          int64_t total, int64_t x, uint32_t lane) {
    const int2 nb3 = stream_bounds(a, m0, depth, total, x + 3);
    const uint32_t nk2 = stream_kk(a, m0, P.b2, lane);
    int4 ni1 = make_int4(0, 0, 0, 0);
    if (P.k1 != ~0u) ni1 = man_ids(a, m0 + P.k1);
    if (x >= 0 && x < total) {
        if (lane == 0) hdr[uint32_t(x) % GIANT_LEVELS] = P.b0;
        if (P.k0 != ~0u) {
            const uint32_t np = P.i0.z < 0 ? 0u : (P.i0.z > 4 ? 4u : uint32_t(P.i0.z));
            GiantSlot* sl = ring + (uint32_t(x) % GIANT_LEVELS) * STREAM_RING + lane;
            sl->desc = make_int4(0, int(np), int(P.k0), P.i0.w);
            const float4* src = a.mrec[m0 + P.k0].q;
            for (int r = 0; r < DQ_ROWS; r++) cp_async16(&sl->mq[r], src + r);
            const float4* ps = a.prec[P.i0.w].q;
            for (uint32_t r = 0; r < np * PREC_F4; r++) cp_async16(&sl->pq[r], ps + r);
        }
    }
    if (x >= 0) cp_async_commit();
    P.b0 = P.b1;
    P.b1 = P.b2;
    P.b2 = nb3;
    P.k0 = P.k1;
    P.k1 = nk2;
    P.i0 = ni1;
}

// Both warps: warm start and velocity iterations of a scheduled island.
RD void stream_solve(const DynArgs& a, uint32_t m0, GiantSlot* ring, uint32_t warp, uint32_t lane, uint32_t depth) {
    const uint32_t total = uint32_t(a.iterations + 1) * depth;
    int2* hdr = reinterpret_cast<int2*>(ring + GIANT_LEVELS * STREAM_RING);
    if (warp == 1) {
        StreamPipe P;
        P.b0 = P.b1 = P.b2 = make_int2(0, 0);
        P.k0 = P.k1 = ~0u;
        P.i0 = make_int4(0, 0, 0, 0);
        for (int64_t x = -3; x <= 1; x++) stream_stage_step(a, ring, hdr, P, m0, depth, total, x, lane);
        cp_async_wait<1>();
        giant_bar();
        for (uint32_t t = 0; t < total; t++) {
            stream_stage_step(a, ring, hdr, P, m0, depth, total, int64_t(t) + 2, lane);
            cp_async_wait<1>();
            giant_bar();
        }
        cp_async_wait<0>();
    } else {
        const float beta = a.split ? BETA_SPLIT_IMPULSE : BETA;
        giant_bar();
        for (uint32_t t = 0; t < total; t++) {
            const bool warm = t < depth;
            const int2 bd = hdr[t % GIANT_LEVELS];
            const uint32_t b = uint32_t(bd.x), e = uint32_t(bd.y);
            if (lane < STREAM_RING && b + lane < e) {
                const GiantSlot* sl = ring + (t % GIANT_LEVELS) * STREAM_RING + lane;
                const int4 d = sl->desc;
                const float4 ids = sl->mq[DQ_IDS];
                const BodyVel bv = vel_global(a, __float_as_int(ids.x), __float_as_int(ids.y));
                RecSrc r;
                r.mq = sl->mq;
                r.pq = sl->pq;
                r.pq_stride = PREC_F4;
                r.mmut = &a.mrec[m0 + uint32_t(d.z)].mut;
                r.pmut = &a.prec[d.w].mut;
                r.pmut_stride = PREC_F4;
                if (warm) warm_core<false, true>(a, r, bv, d.y);
                else solve_core<false, true>(a, r, beta, bv, d.y);
            }
            // manifolds of a level beyond the ring read their rows from global memory
            for (uint32_t j = b + STREAM_RING + lane; j < e; j += 32) {
                const uint32_t mi = m0 + a.order[m0 + j];
                const int4 id = man_ids(a, mi);
                const BodyVel bv = vel_global(a, id.x, id.y);
                if (warm) warm_core<true, true>(a, rec_global(a, mi, id.w), bv, id.z);
                else solve_core<true, true>(a, rec_global(a, mi, id.w), beta, bv, id.z);
            }
            __syncwarp();
            giant_bar();
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(GIANT_THREADS, 1) dyn_islands_giant(const DynArgs a) {
    extern __shared__ __align__(16) unsigned char gsm[];
    __shared__ uint32_t s_island, s_ok, s_depth, s_nslots, s_p0;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n_giant = a.counters[3];
    for (;;) {
        if (threadIdx.x == 0) s_island = atomicAdd(a.counters + 4, 1u);
        __syncthreads();
        const uint32_t k = s_island;
        if (k >= n_giant) break;
        const uint32_t is = a.giant_list[k];
        const uint32_t m0 = a.i_start[is], cnt = a.i_count[is];
        GiantStage g;
        if (warp == 0) {
            uint32_t depth = 0, nslots = 0, p0 = 0;
            const bool ok = giant_schedule(a, m0, cnt, gsm, g, lane, depth, nslots, p0);
            if (lane == 0) { s_ok = ok ? 1u : 0u; s_depth = depth; s_nslots = nslots; s_p0 = p0; }
        }
        __syncthreads();
        if (s_ok) {
            if (warp == 1) {
                // the same layout (a pure function of the island's sizes)
                const int4 l = man_ids(a, m0 + cnt - 1);
                giant_layout(a, cnt, uint32_t(int64_t(l.w) + int64_t(l.z) - int64_t(s_p0)), gsm, g);
            }
            giant_solve(a, m0, cnt, g, warp, lane, s_depth, s_nslots, s_p0);
        } else if (size_t(GIANT_LEVELS) * STREAM_RING * sizeof(GiantSlot) + GIANT_LEVELS * sizeof(int2) <= a.giant_smem) {
            // streamed by dyn_islands_stream (queued at the back of giant_list)
            if (threadIdx.x == 0) a.giant_list[a.ni - 1 - atomicAdd(a.counters + 5, 1u)] = is;
            __syncthreads();
            continue;
        } else if (warp == 0) {
            solve_global(a, m0, cnt, lane);
        }
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < cnt; j += GIANT_THREADS) store_manifold(a, m0 + j);
        __syncthreads();
    }
}

// ---- kernel 3d: islands streamed through global memory -------------------
__global__ void __launch_bounds__(GIANT_THREADS, 1) dyn_islands_stream(const DynArgs a) {
    extern __shared__ __align__(16) unsigned char ssm[];
    __shared__ uint32_t s_island, s_depth;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n_stream = a.counters[5];
    for (;;) {
        if (threadIdx.x == 0) s_island = atomicAdd(a.counters + 6, 1u);
        __syncthreads();
        const uint32_t k = s_island;
        if (k >= n_stream) break;
        const uint32_t is = a.giant_list[a.ni - 1 - k];
        const uint32_t m0 = a.i_start[is], cnt = a.i_count[is];
        if (warp == 0) {
            const uint32_t depth = stream_schedule(a, m0, cnt, lane);
            if (lane == 0) s_depth = depth;
        }
        __syncthreads();
        stream_solve(a, m0, reinterpret_cast<GiantSlot*>(ssm), warp, lane, s_depth);
        for (uint32_t j = threadIdx.x; j < cnt; j += GIANT_THREADS) store_manifold(a, m0 + j);
        __syncthreads();
    }
}

// ---- kernel 4: integrateRigidBodiesPositions + updateBodiesState ----------
__global__ void __launch_bounds__(128) dyn_bodies_post(const DynArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nb || !body_enabled(a, i)) return;
    const float dt = a.dt;
    const float f = a.split ? 1.0f : 0.0f;
    const v3 cv = L3(a.cv[i]), cw = L3(a.cw[i]);
    const v3 sv = L3(a.sv[i]), sw = L3(a.sw[i]);
    const v3 nl = V(cv.x + f * sv.x, cv.y + f * sv.y, cv.z + f * sv.z);
    const v3 na = V(cw.x + f * sw.x, cw.y + f * sw.y, cw.z + f * sw.z);
    const v3 x = L3(a.com_world[i]);
    const float4 o4 = a.orientation[i];
    const quat q = Q(o4.x, o4.y, o4.z, o4.w);
    const v3 cp = V(x.x + dt * nl.x, x.y + dt * nl.y, x.z + dt * nl.z);
    const quat dq = qmul(Q(na.x, na.y, na.z, 0.0f), q);
    const quat sq = Q(dt * (0.5f * dq.x), dt * (0.5f * dq.y), dt * (0.5f * dq.z), dt * (0.5f * dq.w));
    const quat co = Q(q.x + sq.x, q.y + sq.y, q.z + sq.z, q.w + sq.w);
    if (a.xc) {
        // mConstrainedPositions / mConstrainedOrientations, read by the joints' position correction
        a.xc[i] = F4(cp);
        a.qc[i] = make_float4(co.x, co.y, co.z, co.w);
    }
    // updateBodiesState
    a.lin_vel[i] = F4(cv);
    a.ang_vel[i] = F4(cw);
    a.com_world[i] = F4(cp);
    const float len = sqrtf(co.x * co.x + co.y * co.y + co.z * co.z + co.w * co.w);
    const quat u = Q(co.x / len, co.y / len, co.z / len, co.w / len);
    a.orientation[i] = make_float4(u.x, u.y, u.z, u.w);
    const v3 r = qrot(u, L3(a.com_local[i]));
    a.position[i] = F4(V(cp.x - r.x, cp.y - r.y, cp.z - r.z));
}

// ---- kernel 5: collider local-to-world transforms ------------------------
__global__ void __launch_bounds__(128) dyn_colliders(const DynArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nc || !collider_enabled(a, i)) return;
    const int32_t b = a.c_body[i];
    if (uint32_t(b) >= a.nb) {
        atomicOr(a.error, 4u);
        return;
    }
    const float4 bo = a.orientation[b], lo = a.c_lori[i];
    const xform t = xmul(X(L3(a.position[b]), Q(bo.x, bo.y, bo.z, bo.w)), X(L3(a.c_lpos[i]), Q(lo.x, lo.y, lo.z, lo.w)));
    a.c_wpos[i] = F4(t.p);
    a.c_wori[i] = make_float4(t.q.x, t.q.y, t.q.z, t.q.w);
}

uint32_t blocks(uint32_t n) { return (n + 127) / 128; }

// ---- graph-coloured solver -------------------------------------------------
//
// Not the drop-in (the drop-in is the exact-order solver above): for very
// large worlds, where one island of 10^5 manifolds is a chain of 10^4
// dependency levels, the manifolds' conflict graph (two manifolds conflict
// when they share a movable body) is coloured on the GPU and every pass (warm
// start, each velocity iteration) runs colour after colour, the manifolds of
// one colour in parallel.  No two manifolds of a colour share a movable body,
// so each manifold still reads the latest velocities of its bodies and the
// per-manifold arithmetic is the reference's (ContactSolverSystem.cpp:
// 324-759); only the order of the manifolds differs, so the results differ
// from the reference's and the solver is reported by its constraint residual
// and energy, next to the exact solver on the same world.
//
// Colouring: speculative greedy rounds.  Each uncoloured manifold takes the
// lowest colour none of its coloured neighbours has; of two neighbours that
// took the same colour in a round, the one with the lower index keeps it and
// the other tries again in the next round.  Decisions depend on the previous
// round only, so the colouring is deterministic.
constexpr uint8_t NO_COLOR = 0xff;

RD uint32_t movable_mask(const DynArgs& a, uint32_t mi) { return ~man_fixed(a, mi) & 3u; }

__global__ void __launch_bounds__(128) color_degree(const DynArgs a, uint32_t* __restrict__ deg) {
    const uint32_t mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= a.nm) return;
    const int4 id = man_ids(a, mi);
    const uint32_t mv = movable_mask(a, mi);
    if (mv & 1u) atomicAdd(deg + id.x, 1u);
    if (mv & 2u) atomicAdd(deg + id.y, 1u);
}

__global__ void __launch_bounds__(128) color_adjacency(const DynArgs a, const uint32_t* __restrict__ start,
                                                       uint32_t* __restrict__ fill, uint32_t* __restrict__ adj) {
    const uint32_t mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= a.nm) return;
    const int4 id = man_ids(a, mi);
    const uint32_t mv = movable_mask(a, mi);
    if (mv & 1u) adj[start[id.x] + atomicAdd(fill + id.x, 1u)] = mi;
    if (mv & 2u) adj[start[id.y] + atomicAdd(fill + id.y, 1u)] = mi;
}

__global__ void __launch_bounds__(128) color_tentative(const DynArgs a, ColorScratch c) {
    const uint32_t mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= a.nm) return;
    if (c.color[mi] != NO_COLOR) { c.tent[mi] = NO_COLOR; return; }
    const int4 id = man_ids(a, mi);
    const uint32_t mv = movable_mask(a, mi);
    unsigned long long used[2] = {0ull, 0ull};
    for (int side = 0; side < 2; side++) {
        if (!(mv & (1u << side))) continue;
        const int32_t b = side ? id.y : id.x;
        for (uint32_t k = c.start[b]; k < c.start[b + 1]; k++) {
            const uint8_t nc = c.color[c.adj[k]];
            if (nc != NO_COLOR) used[nc >> 6] |= 1ull << (nc & 63u);
        }
    }
    uint8_t t = NO_COLOR;
    if (~used[0]) t = uint8_t(__ffsll(static_cast<long long>(~used[0])) - 1);
    else if (~used[1]) t = uint8_t(64 + __ffsll(static_cast<long long>(~used[1])) - 1);
    c.tent[mi] = t;   // NO_COLOR: every colour is taken (the caller falls back)
}

// Priority of a manifold in the conflict resolution: a hash of its index
// (ties by index).  Index order itself follows the islands, i.e. space, so a
// pile would chain "lower index wins" decisions over hundreds of rounds; a
// hashed order resolves every round's conflicts independently of position
// (a few rounds to colour the 100k-body terrain's island).
RD uint64_t color_priority(uint32_t mi) {
    uint32_t h = mi * 0x9E3779B1u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    return (uint64_t(h) << 32) | mi;
}

__global__ void __launch_bounds__(128) color_resolve(const DynArgs a, ColorScratch c) {
    const uint32_t mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi >= a.nm) return;
    const uint8_t t = c.tent[mi];
    if (t == NO_COLOR) {
        if (c.color[mi] == NO_COLOR) atomicAdd(c.count + COLOR_MAX, 1u);
        return;
    }
    const int4 id = man_ids(a, mi);
    const uint32_t mv = movable_mask(a, mi);
    for (int side = 0; side < 2; side++) {
        if (!(mv & (1u << side))) continue;
        const int32_t b = side ? id.y : id.x;
        for (uint32_t k = c.start[b]; k < c.start[b + 1]; k++) {
            const uint32_t n = c.adj[k];
            if (n != mi && c.tent[n] == t && color_priority(n) < color_priority(mi)) {
                atomicAdd(c.count + COLOR_MAX, 1u);
                return;
            }
        }
    }
    c.color[mi] = t;
}

__global__ void __launch_bounds__(128) color_count(const DynArgs a, ColorScratch c) {
    const uint32_t mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi < a.nm) atomicAdd(c.count + c.color[mi], 1u);
}

// Manifolds grouped by colour (the order inside a colour does not matter:
// its manifolds share no movable body).
__global__ void __launch_bounds__(128) color_scatter(const DynArgs a, ColorScratch c) {
    const uint32_t mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi < a.nm) c.order[atomicAdd(c.offset + c.color[mi], 1u)] = mi;
}

template <int PASS>   // 0 warm start, 1 velocity iteration
__global__ void __launch_bounds__(128) colored_pass(const DynArgs a, const uint32_t* __restrict__ order, uint32_t off,
                                                    uint32_t cnt, float beta) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cnt) return;
    const uint32_t mi = order[off + k];
    const int4 id = man_ids(a, mi);
    if (PASS == 0) warm_manifold(a, mi, vel_global(a, id.x, id.y), id.z, id.w);
    else solve_manifold(a, mi, beta, vel_global(a, id.x, id.y), id.z, id.w);
}

__global__ void __launch_bounds__(128) colored_store(const DynArgs a) {
    const uint32_t mi = blockIdx.x * blockDim.x + threadIdx.x;
    if (mi < a.nm) store_manifold(a, mi);
}

// Velocity constraint residual of every contact point after the solve, on
// the constrained velocities (either solver).
__global__ void __launch_bounds__(128) solver_residual(const DynArgs a) {
    const uint32_t mi = blockIdx.x * blockDim.x + threadIdx.x;
    float sq = 0.0f, mx = 0.0f;
    uint32_t np = 0;
    if (mi < a.nm) {
        const int4 id = man_ids(a, mi);
        const v3 v1 = L3(a.cv[id.x]), w1 = L3(a.cw[id.x]), v2 = L3(a.cv[id.y]), w2 = L3(a.cw[id.y]);
        for (int k = 0; k < id.z; k++) {
            const DynPointRec& pr = a.prec[id.w + k];
            const v3 r1 = L3(pr.q[DP_R1]), r2 = L3(pr.q[DP_R2]), n = L3(pr.q[DP_N]);
            const float jv = vdot(rel_velocity(v1, w1, v2, w2, r1, r2), n);
            const float lambda = pr.mut.x;
            const float r = lambda > 0.0f ? fabsf(jv) : (jv < 0.0f ? -jv : 0.0f);
            sq += r * r;
            mx = fmaxf(mx, r);
            np++;
        }
    }
    for (int o = 16; o; o >>= 1) {
        sq += __shfl_xor_sync(0xffffffffu, sq, o);
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        np += __shfl_xor_sync(0xffffffffu, np, o);
    }
    if ((threadIdx.x & 31u) == 0 && np) {
        atomicAdd(&a.stats->residual_sq_sum, double(sq));
        atomicMax(&a.stats->residual_max_bits, __float_as_uint(mx));
        atomicAdd(&a.stats->points, np);
    }
}

// Energies of the enabled dynamic bodies after the stage.
__global__ void __launch_bounds__(128) body_energy(const DynArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0, pe = 0.0;
    if (i < a.nb && body_enabled(a, i)) {
        const float4 m = a.mass[i];   // mass, inverse mass, dampings
        if (m.y > 0.0f) {
            const v3 v = L3(a.lin_vel[i]), w = L3(a.ang_vel[i]);
            const float4 o = a.orientation[i];
            const v3 wl = qrot(qinv(Q(o.x, o.y, o.z, o.w)), w);   // angular velocity in the body frame
            const v3 ii = L3(a.iil[i]);
            double rot = 0.0;
            if (ii.x > 0.0f) rot += double(wl.x) * wl.x / ii.x;
            if (ii.y > 0.0f) rot += double(wl.y) * wl.y / ii.y;
            if (ii.z > 0.0f) rot += double(wl.z) * wl.z / ii.z;
            ke = 0.5 * double(m.x) * (double(v.x) * v.x + double(v.y) * v.y + double(v.z) * v.z) + 0.5 * rot;
            if (a.gravity_enabled && a.gravity[i]) {
                const float4 x = a.com_world[i];
                pe = -double(m.x) * (double(a.gx) * x.x + double(a.gy) * x.y + double(a.gz) * x.z);
            }
        }
    }
    for (int o = 16; o; o >>= 1) {
        ke += __shfl_xor_sync(0xffffffffu, ke, o);
        pe += __shfl_xor_sync(0xffffffffu, pe, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(&a.stats->kinetic, ke);
        atomicAdd(&a.stats->potential, pe);
    }
}

// Colours every manifold and runs the passes; false when the colouring does
// not finish (every colour taken around some manifold, or too many rounds):
// the caller then runs the exact solver.  Synchronizes the stream.
bool colored_islands(const DynArgs& a, cudaStream_t s, uint64_t* launches) {
    ColorScratch c = *a.color;
    const uint32_t nm = a.nm;
    cudaMemsetAsync(c.start, 0, (size_t(a.nb) + 1) * 4, s);
    cudaMemsetAsync(c.fill, 0, size_t(a.nb) * 4, s);
    cudaMemsetAsync(c.color, NO_COLOR, nm, s);
    color_degree<<<blocks(nm), 128, 0, s>>>(a, c.start);
    launch_exclusive_scan(c.start, a.nb + 1, nullptr, s);
    color_adjacency<<<blocks(nm), 128, 0, s>>>(a, c.start, c.fill, c.adj);
    *launches += 3;
    uint32_t rounds = 0, remaining = nm;
    while (remaining > 0) {
        if (++rounds > 256) return false;
        cudaMemsetAsync(c.count + COLOR_MAX, 0, 4, s);
        color_tentative<<<blocks(nm), 128, 0, s>>>(a, c);
        color_resolve<<<blocks(nm), 128, 0, s>>>(a, c);
        *launches += 2;
        if (cudaMemcpyAsync(&remaining, c.count + COLOR_MAX, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return false;
        // (a manifold whose neighbours hold every colour never gets one: the
        // round limit ends the loop)
    }
    uint32_t cnt[COLOR_MAX];
    cudaMemsetAsync(c.count, 0, COLOR_MAX * 4, s);
    color_count<<<blocks(nm), 128, 0, s>>>(a, c);
    *launches += 1;
    if (cudaMemcpyAsync(cnt, c.count, sizeof(cnt), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return false;
    uint32_t off[COLOR_MAX], ncol = 0, run = 0;
    for (uint32_t k = 0; k < COLOR_MAX; k++) {
        off[k] = run;
        run += cnt[k];
        if (cnt[k]) ncol = k + 1;
    }
    cudaMemcpyAsync(c.offset, off, sizeof(off), cudaMemcpyHostToDevice, s);
    color_scatter<<<blocks(nm), 128, 0, s>>>(a, c);
    *launches += 1;
    const float beta = a.split ? BETA_SPLIT_IMPULSE : BETA;
    for (uint32_t k = 0; k < ncol; k++)
        if (cnt[k]) { colored_pass<0><<<blocks(cnt[k]), 128, 0, s>>>(a, c.order, off[k], cnt[k], beta); (*launches)++; }
    for (int it = 0; it < a.iterations; it++)
        for (uint32_t k = 0; k < ncol; k++)
            if (cnt[k]) { colored_pass<1><<<blocks(cnt[k]), 128, 0, s>>>(a, c.order, off[k], cnt[k], beta); (*launches)++; }
    colored_store<<<blocks(nm), 128, 0, s>>>(a);
    (*launches)++;
    if (a.stats) {
        uint32_t cr[2] = {ncol, rounds};
        cudaMemcpyAsync(&a.stats->colors, cr, sizeof(cr), cudaMemcpyHostToDevice, s);
        // the pageable source is read before the function returns
        cudaStreamSynchronize(s);
    }
    return true;
}

}  // namespace

cudaError_t launch_dynamics(const DynArgs& a, cudaStream_t s, uint64_t* launches) {
    if (a.nb) { dyn_bodies_pre<<<blocks(a.nb), 128, 0, s>>>(a); (*launches)++; }
    if (a.nm) { dyn_manifold_init<<<blocks(a.nm), 128, 0, s>>>(a); (*launches)++; }
    if (a.nj) { dyn_joints_init<<<blocks(a.nj), 128, 0, s>>>(a); (*launches)++; }
    if (a.stats) cudaMemsetAsync(a.stats, 0, sizeof(SolverStats), s);
    // the graph-coloured solver takes every island when the stage has no
    // joints (joint islands keep the exact order); it falls back to the exact
    // solver if the colouring does not finish
    bool colored_done = false;
    if (a.colored && a.color && a.nj == 0 && a.nm) colored_done = colored_islands(a, s, launches);
    if (a.ni && !colored_done) {
        cudaMemsetAsync(a.counters, 0, 7 * sizeof(uint32_t), s);
        dyn_islands_small<<<blocks(a.ni), 128, 0, s>>>(a);
        (*launches)++;
        const size_t smem = size_t(LARGE_WARPS) * LARGE_WARP_SMEM;
        cudaFuncSetAttribute(dyn_islands_large, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        dyn_islands_large<<<a.large_ctas, LARGE_WARPS * 32, smem, s>>>(a);
        (*launches)++;
        if (a.giant_smem) {
            cudaFuncSetAttribute(dyn_islands_giant, cudaFuncAttributeMaxDynamicSharedMemorySize, int(a.giant_smem));
            dyn_islands_giant<<<a.giant_ctas, GIANT_THREADS, a.giant_smem, s>>>(a);
            (*launches)++;
            const size_t ring = size_t(GIANT_LEVELS) * STREAM_RING * sizeof(GiantSlot) + GIANT_LEVELS * sizeof(int2);
            cudaFuncSetAttribute(dyn_islands_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ring));
            dyn_islands_stream<<<a.giant_ctas, GIANT_THREADS, ring, s>>>(a);
            (*launches)++;
        }
        if (a.nji) { dyn_islands_joint<<<(a.nji + 63) / 64, 64, 0, s>>>(a); (*launches)++; }
    }
    if (a.stats && a.nm) { solver_residual<<<blocks(a.nm), 128, 0, s>>>(a); (*launches)++; }
    const uint32_t nbp = a.b_enabled ? a.nb : a.nb_enabled, ncp = a.c_enabled ? a.nc : a.nc_enabled;
    if (nbp) { dyn_bodies_post<<<blocks(nbp), 128, 0, s>>>(a); (*launches)++; }
    if (a.stats && a.nb) { body_energy<<<blocks(a.nb), 128, 0, s>>>(a); (*launches)++; }
    if (a.nji) { dyn_joints_position<<<(a.nji + 63) / 64, 64, 0, s>>>(a); (*launches)++; }
    if (ncp) { dyn_colliders<<<blocks(ncp), 128, 0, s>>>(a); (*launches)++; }
    return cudaGetLastError();
}

}  // namespace rp3dg
