// reduceContactPoints (reference src/systems/CollisionDetectionSystem.cpp:
// 1483-1662) and removeDuplicatedContactPointsInManifold (:1673-1705) over a
// manifold's list of point ids; lp1[id] gives the point on shape 1 in
// shape-1 local space.  Used by the convex manifold step (one manifold per
// pair, at most 16 points) and the concave one (up to 255 points).
#pragma once
#include "rp3dg_math.cuh"

namespace rp3dg {

constexpr float SAME_POINT_DIST = 0.01f;  // SAME_CONTACT_POINT_DISTANCE_THRESHOLD, configuration.h:146

// points held in a local array
struct LocalPoints {
    const v3* p;
    RD v3 operator[](uint32_t i) const { return p[i]; }
};

RD void remove_at(uint32_t* a, uint32_t idx, uint32_t& size) { a[idx] = a[size - 1]; size--; }

// reduceContactPoints: idx holds the manifold's points (nb > 4), 4 on exit;
// cand is scratch for nb entries.
template <class LP>
RD void reduce_points(uint32_t* idx, uint32_t& nb, const LP& lp1, v3 normal0, quat q1, uint32_t* cand) {
    uint32_t ncand = nb;
    for (uint32_t i = 0; i < ncand; i++) cand[i] = idx[i];
    uint32_t keep[4] = {0, 0, 0, 0};
    // contact normal in shape-1 space: worldToShape1.getOrientation() = conjugate
    const v3 nLocal = qrot(qinv(q1), normal0);
    float maxDot = DECIMAL_SMALLEST;
    uint32_t k = 0;
    for (uint32_t i = 0; i < ncand; i++) {
        const float d = vdot(V(1.0f, 1.0f, 1.0f), lp1[cand[i]]);
        if (d > maxDot) { maxDot = d; k = i; }
    }
    keep[0] = cand[k];
    remove_at(cand, k, ncand);
    float maxDist = 0.0f;
    k = 0;
    for (uint32_t i = 0; i < ncand; i++) {
        const float d = vlen2(vsub(lp1[keep[0]], lp1[cand[i]]));
        if (d >= maxDist) { maxDist = d; k = i; }
    }
    keep[1] = cand[k];
    remove_at(cand, k, ncand);
    uint32_t kmax = 0, kmin = 0;
    float minArea = 0.0f, maxArea = 0.0f;
    bool prevPositive;
    for (uint32_t i = 0; i < ncand; i++) {
        const v3 a = vsub(lp1[keep[0]], lp1[cand[i]]);
        const v3 b = vsub(lp1[keep[1]], lp1[cand[i]]);
        const float area = vdot(vcross(a, b), nLocal);
        if (area >= maxArea) { maxArea = area; kmax = i; }
        if (area <= minArea) { minArea = area; kmin = i; }
    }
    if (maxArea > (-minArea)) { prevPositive = true; keep[2] = cand[kmax]; remove_at(cand, kmax, ncand); }
    else { prevPositive = false; keep[2] = cand[kmin]; remove_at(cand, kmin, ncand); }
    float largest = 0.0f;
    k = 0;
    for (uint32_t i = 0; i < ncand; i++) {
        for (uint32_t j = 0; j < 3; j++) {
            const uint32_t e1 = j, e2 = j < 2 ? j + 1 : 0;
            const v3 a = vsub(lp1[keep[e1]], lp1[cand[i]]);
            const v3 b = vsub(lp1[keep[e2]], lp1[cand[i]]);
            const float area = vdot(vcross(a, b), nLocal);
            if (prevPositive && area <= largest) { largest = area; k = i; }
            else if (!prevPositive && area >= largest) { largest = area; k = i; }
        }
    }
    keep[3] = cand[k];
    for (int i = 0; i < 4; i++) idx[i] = keep[i];
    nb = 4;
}

// removeDuplicatedContactPointsInManifold
template <class LP>
RD void remove_duplicates(uint32_t* idx, uint32_t& nb, const LP& lp1) {
    const float thr = SAME_POINT_DIST * SAME_POINT_DIST;
    for (uint32_t i = 0; i < nb; i++) {
        for (uint32_t j = i + 1; j < nb; j++) {
            if (vlen2(vsub(lp1[idx[j]], lp1[idx[i]])) < thr) {
                idx[j] = idx[nb - 1];
                nb--;
                j--;
            }
        }
    }
}

}  // namespace rp3dg
