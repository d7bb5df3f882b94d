// CollisionShape::computeTransformedAABB (reference
// src/collision/shapes/CollisionShape.cpp:54-90) with the sphere override
// (SphereShape.cpp:49-58), shared by the broad phase (world AABBs) and the
// convex vs concave middle phase (convex AABB in the concave shape's space).
#pragma once
#include "../../include/rp3dg.h"
#include "rp3dg_math.cuh"

namespace rp3dg {

// Quaternion::getMatrix (src/mathematics/Quaternion.cpp:138-165)
RD void quat_matrix_aabb(quat q, float* r) {
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

// AABB of a shape (kind, sphere radius, local bounds lo / hi) under transform t.
RD void shape_transformed_aabb(int kind, float radius, float4 lo, float4 hi, const xform& t, v3& amin, v3& amax) {
    if (kind == RP3DG_SHAPE_SPHERE) {
        // SphereShape::computeTransformedAABB: position -/+ (margin, margin, margin)
        amin = V(t.p.x - radius, t.p.y - radius, t.p.z - radius);
        amax = V(t.p.x + radius, t.p.y + radius, t.p.z + radius);
        return;
    }
    const float bmin[3] = {lo.x, lo.y, lo.z}, bmax[3] = {hi.x, hi.y, hi.z}, tt[3] = {t.p.x, t.p.y, t.p.z};
    float m[9];
    quat_matrix_aabb(t.q, m);
    float rmin[3], rmax[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        rmin[r] = tt[r];
        rmax[r] = tt[r];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float e = m[3 * r + c] * bmin[c];
            const float f = m[3 * r + c] * bmax[c];
            if (e < f) { rmin[r] += e; rmax[r] += f; }
            else { rmin[r] += f; rmax[r] += e; }
        }
    }
    amin = V(rmin[0], rmin[1], rmin[2]);
    amax = V(rmax[0], rmax[1], rmax[2]);
}

}  // namespace rp3dg
