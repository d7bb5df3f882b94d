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

#include "dynamics_launch.h"
#include "rp3dg_math.cuh"

namespace rp3dg {

namespace {

constexpr float BETA = 0.2f;               // ContactSolverSystem.cpp:43
constexpr float BETA_SPLIT_IMPULSE = 0.2f;  // :44
constexpr float SLOP = 0.01f;              // :45

RD v3 L3(const float4 a) { return V(a.x, a.y, a.z); }
RD float4 F4(v3 a, float w = 0.0f) { return make_float4(a.x, a.y, a.z, w); }
RD v3 A3(const float* a) { return V(a[0], a[1], a[2]); }
RD void S3(float* a, v3 v) { a[0] = v.x; a[1] = v.y; a[2] = v.z; }

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

// ---- kernel 1: world inverse inertia + velocity integration --------------
__global__ void __launch_bounds__(128) dyn_bodies_pre(const DynArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nb) return;
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    a.sv[i] = zero;
    a.sw[i] = zero;
    if (i >= a.nb_enabled) {
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

RD void load_rows(const float4* rows, float* I) {
    const float4 r0 = rows[0], r1 = rows[1], r2 = rows[2];
    I[0] = r0.x; I[1] = r0.y; I[2] = r0.z;
    I[3] = r1.x; I[4] = r1.y; I[5] = r1.z;
    I[6] = r2.x; I[7] = r2.y; I[8] = r2.z;
}

RD bool is_fixed(const DynArgs& a, int32_t b) {
    if (uint32_t(b) >= a.nb_enabled) return true;
    const float4 il = a.iil[b];
    return a.mass[b].y == 0.0f && il.x == 0.0f && il.y == 0.0f && il.z == 0.0f;
}

// ---- kernel 2: ContactSolverSystem::initializeForIsland per manifold ------
// (ContactSolverSystem.cpp:116-318)
__global__ void __launch_bounds__(128) dyn_manifold_init(const DynArgs a) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.nm) return;
    DynManifoldRec& c = a.mrec[m];
    const int4 id = a.m_ids[m];
    const int32_t b1 = id.x, b2 = id.y;
    const uint32_t nb = a.m_npts[m], ps = a.m_pstart[m];
    if (uint32_t(b1) >= a.nb || uint32_t(b2) >= a.nb || b1 == b2 || uint32_t(id.z) >= a.nc ||
        uint32_t(id.w) >= a.nc || nb == 0 || nb > 4 || ps > a.np || nb > a.np - ps) {
        atomicOr(a.error, 4u);
        c.b1 = 0; c.b2 = 0; c.nb = 0; c.pstart = 0; c.fixed_mask = 3.0f;  // solver skips it
        return;
    }
    c.b1 = b1; c.b2 = b2; c.nb = int32_t(nb); c.pstart = int32_t(ps);
    const v3 x1 = L3(a.com_world[b1]), x2 = L3(a.com_world[b2]);
    load_rows(a.iiw + 3 * b1, c.I1);
    load_rows(a.iiw + 3 * b2, c.I2);
    c.im1 = a.mass[b1].y;
    c.im2 = a.mass[b2].y;
    S3(c.lf1, L3(a.llock[b1])); S3(c.lf2, L3(a.llock[b2]));
    S3(c.alf1, L3(a.alock[b1])); S3(c.alf2, L3(a.alock[b2]));
    c.fixed_mask = float((is_fixed(a, b1) ? 1 : 0) | (is_fixed(a, b2) ? 2 : 0));
    const float4 mat1 = a.c_mat[id.z], mat2 = a.c_mat[id.w];
    c.friction = mat1.x * mat2.x;                          // computeMixedFrictionCoefficient
    const float restitution = (mat1.y > mat2.y) ? mat1.y : mat2.y;  // computeMixedRestitutionFactor
    const v3 v1 = L3(a.lin_vel[b1]), w1 = L3(a.ang_vel[b1]);
    const v3 v2 = L3(a.lin_vel[b2]), w2 = L3(a.ang_vel[b2]);
    const xform t1 = X(L3(a.c_wpos[id.z]), Q(a.c_wori[id.z].x, a.c_wori[id.z].y, a.c_wori[id.z].z, a.c_wori[id.z].w));
    const xform t2 = X(L3(a.c_wpos[id.w]), Q(a.c_wori[id.w].x, a.c_wori[id.w].y, a.c_wori[id.w].z, a.c_wori[id.w].w));
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
        S3(r.r1, r1); S3(r.r2, r2); S3(r.normal, n);
        r.depth = nd.w;
        r.resting = a.p_resting[p];
        a.p_resting[p] = 1;
        r.impulse = a.p_impulse[p];
        r.split_impulse = 0.0f;
        fp1 = V(fp1.x + p1.x, fp1.y + p1.y, fp1.z + p1.z);
        fp2 = V(fp2.x + p2.x, fp2.y + p2.y, fp2.z + p2.z);
        const v3 dv = rel_velocity(v1, w1, v2, w2, r1, r2);
        const v3 r1n = vcross(r1, n), r2n = vcross(r2, n);
        const v3 i1 = mv(c.I1, r1n), i2 = mv(c.I2, r2n);
        S3(r.i1, i1); S3(r.i2, i2);
        const float mp = c.im1 + c.im2 + vdot(vcross(i1, r1), n) + vdot(vcross(i2, r2), n);
        r.inv_mass = mp > 0.0f ? 1.0f / mp : 0.0f;
        r.restitution_bias = 0.0f;
        const float dvn = dv.x * n.x + dv.y * n.y + dv.z * n.z;
        if (dvn < -a.restitution_threshold) r.restitution_bias = restitution * dvn;
        nsum = V(nsum.x + n.x, nsum.y + n.y, nsum.z + n.z);
    }
    const float fnb = float(nb);
    fp1 = vdivs(fp1, fnb);
    fp2 = vdivs(fp2, fnb);
    const v3 r1f = V(fp1.x - x1.x, fp1.y - x1.y, fp1.z - x1.z);
    const v3 r2f = V(fp2.x - x2.x, fp2.y - x2.y, fp2.z - x2.z);
    S3(c.r1f, r1f); S3(c.r2f, r2f);
    S3(c.ofv1, L3(a.m_fv1[m]));
    S3(c.ofv2, L3(a.m_fv2[m]));
    const float4 fi = a.m_fimp[m];
    c.f1 = fi.x; c.f2 = fi.y; c.ftw = fi.z;
    const v3 n = vnormalize(nsum);
    S3(c.normal, n);
    // computeFrictionVectors (:789-818)
    const v3 dvf = rel_velocity(v1, w1, v2, w2, r1f, r2f);
    const float dvfn = vdot(dvf, n);
    const v3 nv = vmul(n, dvfn);
    const v3 tv = V(dvf.x - nv.x, dvf.y - nv.y, dvf.z - nv.z);
    const float lt = vlen(tv);
    const v3 fv1 = lt > MACHINE_EPSILON ? vdivs(tv, lt) : unit_orthogonal(n);
    const v3 fv2 = vcross(n, fv1);
    S3(c.fv1, fv1); S3(c.fv2, fv2);
    const v3 r1ct1 = vcross(r1f, fv1), r1ct2 = vcross(r1f, fv2);
    const v3 r2ct1 = vcross(r2f, fv1), r2ct2 = vcross(r2f, fv2);
    S3(c.r1ct1, r1ct1); S3(c.r1ct2, r1ct2); S3(c.r2ct1, r2ct1); S3(c.r2ct2, r2ct2);
    const float f1m = c.im1 + c.im2 + vdot(vcross(mv(c.I1, r1ct1), r1f), fv1) + vdot(vcross(mv(c.I2, r2ct1), r2f), fv1);
    const float f2m = c.im1 + c.im2 + vdot(vcross(mv(c.I1, r1ct2), r1f), fv2) + vdot(vcross(mv(c.I2, r2ct2), r2f), fv2);
    const float twm = vdot(n, mv(c.I1, n)) + vdot(n, mv(c.I2, n));
    c.inv_f1 = f1m > 0.0f ? 1.0f / f1m : 0.0f;
    c.inv_f2 = f2m > 0.0f ? 1.0f / f2m : 0.0f;
    c.inv_tw = twm > 0.0f ? 1.0f / twm : 0.0f;
}

// Body velocities of one island's thread (cached loads / stores; the two
// bodies of a manifold are distinct).
struct Vel {
    v3 v1, w1, v2, w2;
};

RD void apply_linear(v3& v, float im, v3 imp, const float* lf, float sign) {
    // v -= im * imp * lf (sign -1) or v += ... (sign +1), per component
    if (sign < 0.0f) v = V(v.x - im * imp.x * lf[0], v.y - im * imp.y * lf[1], v.z - im * imp.z * lf[2]);
    else v = V(v.x + im * imp.x * lf[0], v.y + im * imp.y * lf[1], v.z + im * imp.z * lf[2]);
}

// ---- kernel 3: warm start, velocity iterations, stored impulses ----------
// One thread per island (ContactSolverSystem.cpp:324-785).
__global__ void __launch_bounds__(128) dyn_island_solve(const DynArgs a) {
    const uint32_t is = blockIdx.x * blockDim.x + threadIdx.x;
    if (is >= a.ni) return;
    const uint32_t m0 = a.i_start[is], cnt = a.i_count[is];
    if (m0 > a.nm || cnt > a.nm - m0) {
        atomicOr(a.error, 4u);
        return;
    }
    const uint32_t m1 = m0 + cnt;
    float4* __restrict__ cv = a.cv;
    float4* __restrict__ cw = a.cw;

    // warmStart (:324-476)
    for (uint32_t mi = m0; mi < m1; mi++) {
        DynManifoldRec& c = a.mrec[mi];
        if (c.nb == 0) continue;  // rejected by the manifold kernel
        const int32_t b1 = c.b1, b2 = c.b2;
        const uint32_t fixed = uint32_t(c.fixed_mask);
        v3 v1 = L3(cv[b1]), w1 = L3(cw[b1]), v2 = L3(cv[b2]), w2 = L3(cw[b2]);
        bool resting_any = false;
        for (int k = 0; k < c.nb; k++) {
            DynPointRec& p = a.prec[c.pstart + k];
            if (p.resting) {
                resting_any = true;
                const v3 n = A3(p.normal);
                const float pi = p.impulse;
                const v3 ip = V(n.x * pi, n.y * pi, n.z * pi);
                apply_linear(v1, c.im1, ip, c.lf1, -1.0f);
                w1 = V(w1.x - p.i1[0] * c.alf1[0] * pi, w1.y - p.i1[1] * c.alf1[1] * pi, w1.z - p.i1[2] * c.alf1[2] * pi);
                apply_linear(v2, c.im2, ip, c.lf2, 1.0f);
                w2 = V(w2.x + p.i2[0] * c.alf2[0] * pi, w2.y + p.i2[1] * c.alf2[1] * pi, w2.z + p.i2[2] * c.alf2[2] * pi);
            } else {
                p.impulse = 0.0f;
            }
        }
        if (resting_any) {
            const v3 o1 = A3(c.ofv1), o2 = A3(c.ofv2);
            const v3 ofi = V(c.f1 * o1.x + c.f2 * o2.x, c.f1 * o1.y + c.f2 * o2.y, c.f1 * o1.z + c.f2 * o2.z);
            c.f1 = vdot(ofi, A3(c.fv1));
            c.f2 = vdot(ofi, A3(c.fv2));
            // first friction constraint
            v3 ai1 = V(-c.r1ct1[0] * c.f1, -c.r1ct1[1] * c.f1, -c.r1ct1[2] * c.f1);
            v3 li2 = V(c.fv1[0] * c.f1, c.fv1[1] * c.f1, c.fv1[2] * c.f1);
            v3 ai2 = V(c.r2ct1[0] * c.f1, c.r2ct1[1] * c.f1, c.r2ct1[2] * c.f1);
            apply_linear(v1, c.im1, li2, c.lf1, -1.0f);
            w1 = vadd(w1, vcmul(A3(c.alf1), mv(c.I1, ai1)));
            apply_linear(v2, c.im2, li2, c.lf2, 1.0f);
            w2 = vadd(w2, vcmul(A3(c.alf2), mv(c.I2, ai2)));
            // second friction constraint
            ai1 = V(-c.r1ct2[0] * c.f2, -c.r1ct2[1] * c.f2, -c.r1ct2[2] * c.f2);
            li2 = V(c.fv2[0] * c.f2, c.fv2[1] * c.f2, c.fv2[2] * c.f2);
            ai2 = V(c.r2ct2[0] * c.f2, c.r2ct2[1] * c.f2, c.r2ct2[2] * c.f2);
            apply_linear(v1, c.im1, li2, c.lf1, -1.0f);
            w1 = vadd(w1, vcmul(A3(c.alf1), mv(c.I1, ai1)));
            apply_linear(v2, c.im2, li2, c.lf2, 1.0f);
            w2 = vadd(w2, vcmul(A3(c.alf2), mv(c.I2, ai2)));
            // twist friction constraint (the reference applies the body-2
            // angular impulse to both bodies a second time, :461-465)
            ai1 = V(-c.normal[0] * c.ftw, -c.normal[1] * c.ftw, -c.normal[2] * c.ftw);
            ai2 = V(c.normal[0] * c.ftw, c.normal[1] * c.ftw, c.normal[2] * c.ftw);
            w1 = vadd(w1, vcmul(A3(c.alf1), mv(c.I1, ai1)));
            w2 = vadd(w2, vcmul(A3(c.alf2), mv(c.I2, ai2)));
            w1 = vsub(w1, vcmul(A3(c.alf1), mv(c.I1, ai2)));
            w2 = vadd(w2, vcmul(A3(c.alf2), mv(c.I2, ai2)));
        } else {
            c.f1 = 0.0f; c.f2 = 0.0f; c.ftw = 0.0f;
        }
        if (!(fixed & 1)) { cv[b1] = F4(v1); cw[b1] = F4(w1); }
        if (!(fixed & 2)) { cv[b2] = F4(v2); cw[b2] = F4(w2); }
    }

    // solve (:479-759), iterations x island manifolds in order
    const float beta = a.split ? BETA_SPLIT_IMPULSE : BETA;
    float4* __restrict__ sv = a.sv;
    float4* __restrict__ sw = a.sw;
    for (int it = 0; it < a.iterations; it++) {
        for (uint32_t mi = m0; mi < m1; mi++) {
            DynManifoldRec& c = a.mrec[mi];
            if (c.nb == 0) continue;
            const int32_t b1 = c.b1, b2 = c.b2;
            const uint32_t fixed = uint32_t(c.fixed_mask);
            v3 v1 = L3(cv[b1]), w1 = L3(cw[b1]), v2 = L3(cv[b2]), w2 = L3(cw[b2]);
            v3 s1 = L3(sv[b1]), t1 = L3(sw[b1]), s2 = L3(sv[b2]), t2 = L3(sw[b2]);
            float sum_pen = 0.0f;
            for (int k = 0; k < c.nb; k++) {
                DynPointRec& p = a.prec[c.pstart + k];
                const v3 n = A3(p.normal), r1 = A3(p.r1), r2 = A3(p.r2);
                const v3 dv = rel_velocity(v1, w1, v2, w2, r1, r2);
                const float Jv = dv.x * n.x + dv.y * n.y + dv.z * n.z;
                float bias_pen = 0.0f;
                if (p.depth > SLOP) {
                    const float excess = p.depth - SLOP;
                    bias_pen = -(beta / a.dt) * ((0.0f < excess) ? excess : 0.0f);
                }
                const float b = bias_pen + p.restitution_bias;
                float dl = a.split ? -(Jv + p.restitution_bias) * p.inv_mass : -(Jv + b) * p.inv_mass;
                const float lt = p.impulse;
                const float sum = p.impulse + dl;
                p.impulse = (sum < 0.0f) ? 0.0f : sum;
                dl = p.impulse - lt;
                const v3 li = V(n.x * dl, n.y * dl, n.z * dl);
                apply_linear(v1, c.im1, li, c.lf1, -1.0f);
                w1 = V(w1.x - p.i1[0] * c.alf1[0] * dl, w1.y - p.i1[1] * c.alf1[1] * dl, w1.z - p.i1[2] * c.alf1[2] * dl);
                apply_linear(v2, c.im2, li, c.lf2, 1.0f);
                w2 = V(w2.x + p.i2[0] * c.alf2[0] * dl, w2.y + p.i2[1] * c.alf2[1] * dl, w2.z + p.i2[2] * c.alf2[2] * dl);
                sum_pen += p.impulse;
                if (a.split) {
                    const v3 dvs = rel_velocity(s1, t1, s2, t2, r1, r2);
                    const float Jvs = dvs.x * n.x + dvs.y * n.y + dvs.z * n.z;
                    float dls = -(Jvs + bias_pen) * p.inv_mass;
                    const float lts = p.split_impulse;
                    const float ss = p.split_impulse + dls;
                    p.split_impulse = (ss < 0.0f) ? 0.0f : ss;
                    dls = p.split_impulse - lts;
                    const v3 lis = V(n.x * dls, n.y * dls, n.z * dls);
                    apply_linear(s1, c.im1, lis, c.lf1, -1.0f);
                    t1 = V(t1.x - p.i1[0] * c.alf1[0] * dls, t1.y - p.i1[1] * c.alf1[1] * dls,
                           t1.z - p.i1[2] * c.alf1[2] * dls);
                    apply_linear(s2, c.im2, lis, c.lf2, 1.0f);
                    t2 = V(t2.x + p.i2[0] * c.alf2[0] * dls, t2.y + p.i2[1] * c.alf2[1] * dls,
                           t2.z + p.i2[2] * c.alf2[2] * dls);
                }
            }
            const v3 r1f = A3(c.r1f), r2f = A3(c.r2f);
            // first friction constraint
            {
                const v3 dv = rel_velocity(v1, w1, v2, w2, r1f, r2f);
                const float Jv = dv.x * c.fv1[0] + dv.y * c.fv1[1] + dv.z * c.fv1[2];
                float dl = -Jv * c.inv_f1;
                const float limit = c.friction * sum_pen;
                const float lt = c.f1;
                c.f1 = smax(-limit, smin(c.f1 + dl, limit));
                dl = c.f1 - lt;
                const v3 ai1 = V(-c.r1ct1[0] * dl, -c.r1ct1[1] * dl, -c.r1ct1[2] * dl);
                const v3 li2 = V(c.fv1[0] * dl, c.fv1[1] * dl, c.fv1[2] * dl);
                const v3 ai2 = V(c.r2ct1[0] * dl, c.r2ct1[1] * dl, c.r2ct1[2] * dl);
                apply_linear(v1, c.im1, li2, c.lf1, -1.0f);
                w1 = vadd(w1, vcmul(A3(c.alf1), mv(c.I1, ai1)));
                apply_linear(v2, c.im2, li2, c.lf2, 1.0f);
                w2 = vadd(w2, vcmul(A3(c.alf2), mv(c.I2, ai2)));
            }
            // second friction constraint
            {
                const v3 dv = rel_velocity(v1, w1, v2, w2, r1f, r2f);
                const float Jv = dv.x * c.fv2[0] + dv.y * c.fv2[1] + dv.z * c.fv2[2];
                float dl = -Jv * c.inv_f2;
                const float limit = c.friction * sum_pen;
                const float lt = c.f2;
                c.f2 = smax(-limit, smin(c.f2 + dl, limit));
                dl = c.f2 - lt;
                const v3 ai1 = V(-c.r1ct2[0] * dl, -c.r1ct2[1] * dl, -c.r1ct2[2] * dl);
                const v3 li2 = V(c.fv2[0] * dl, c.fv2[1] * dl, c.fv2[2] * dl);
                const v3 ai2 = V(c.r2ct2[0] * dl, c.r2ct2[1] * dl, c.r2ct2[2] * dl);
                apply_linear(v1, c.im1, li2, c.lf1, -1.0f);
                w1 = vadd(w1, vcmul(A3(c.alf1), mv(c.I1, ai1)));
                apply_linear(v2, c.im2, li2, c.lf2, 1.0f);
                w2 = vadd(w2, vcmul(A3(c.alf2), mv(c.I2, ai2)));
            }
            // twist friction constraint
            {
                const v3 dw = vsub(w2, w1);
                const float Jv = dw.x * c.normal[0] + dw.y * c.normal[1] + dw.z * c.normal[2];
                float dl = -Jv * c.inv_tw;
                const float limit = c.friction * sum_pen;
                const float lt = c.ftw;
                c.ftw = smax(-limit, smin(c.ftw + dl, limit));
                dl = c.ftw - lt;
                const v3 ai2 = V(c.normal[0] * dl, c.normal[1] * dl, c.normal[2] * dl);
                w1 = vsub(w1, vcmul(A3(c.alf1), mv(c.I1, ai2)));
                w2 = vadd(w2, vcmul(A3(c.alf2), mv(c.I2, ai2)));
            }
            if (!(fixed & 1)) { cv[b1] = F4(v1); cw[b1] = F4(w1); sv[b1] = F4(s1); sw[b1] = F4(t1); }
            if (!(fixed & 2)) { cv[b2] = F4(v2); cw[b2] = F4(w2); sv[b2] = F4(s2); sw[b2] = F4(t2); }
        }
    }

    // storeImpulses (:763-785)
    for (uint32_t mi = m0; mi < m1; mi++) {
        const DynManifoldRec& c = a.mrec[mi];
        if (c.nb == 0) continue;
        for (int k = 0; k < c.nb; k++) a.p_impulse[c.pstart + k] = a.prec[c.pstart + k].impulse;
        a.m_fimp[mi] = make_float4(c.f1, c.f2, c.ftw, 0.0f);
        a.m_fv1[mi] = F4(A3(c.fv1));
        a.m_fv2[mi] = F4(A3(c.fv2));
    }
}

// ---- kernel 4: integrateRigidBodiesPositions + updateBodiesState ----------
__global__ void __launch_bounds__(128) dyn_bodies_post(const DynArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nb_enabled) return;
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
    if (i >= a.nc_enabled) return;
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

}  // namespace

cudaError_t launch_dynamics(const DynArgs& a, cudaStream_t s, uint64_t* launches) {
    if (a.nb) { dyn_bodies_pre<<<blocks(a.nb), 128, 0, s>>>(a); (*launches)++; }
    if (a.nm) { dyn_manifold_init<<<blocks(a.nm), 128, 0, s>>>(a); (*launches)++; }
    if (a.ni) { dyn_island_solve<<<blocks(a.ni), 128, 0, s>>>(a); (*launches)++; }
    if (a.nb_enabled) { dyn_bodies_post<<<blocks(a.nb_enabled), 128, 0, s>>>(a); (*launches)++; }
    if (a.nc_enabled) { dyn_colliders<<<blocks(a.nc_enabled), 128, 0, s>>>(a); (*launches)++; }
    return cudaGetLastError();
}

}  // namespace rp3dg
