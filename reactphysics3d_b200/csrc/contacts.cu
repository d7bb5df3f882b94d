// Contact manifolds of convex pairs: the narrow phase's raw points of a
// colliding pair form one manifold (CollisionDetectionSystem::
// processPotentialContacts, reference src/systems/CollisionDetectionSystem.cpp:
// 1198-1391, convex branch), which is reduced to at most 4 points when it has
// more (reduceContactPoints, :1483-1662) and de-duplicated
// (removeDuplicatedContactPointsInManifold, :1673-1705), as
// reducePotentialContactManifolds does (:1394-1458).  One pair per thread; the
// kept points are compacted in place into the first contact slots.
#include <cuda_runtime.h>

#include "contacts_launch.h"
#include "rp3dg_math.cuh"
#include "manifold_reduce.cuh"

namespace rp3dg {

constexpr uint32_t MAX_RAW = RP3DG_MAX_CONTACTS_PER_PAIR;

__global__ void __launch_bounds__(128) contacts_reduce_kernel(const ReduceArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const bool colliding = a.is_colliding[i] != 0;
    if (a.cache) {
        // processPotentialContacts (:1209-1217): the last-frame info becomes
        // valid and remembers whether the pair collided
        uint8_t& f = a.cache[i].flags;
        f = uint8_t((f | RP3DG_LF_IS_VALID) & ~RP3DG_LF_WAS_COLLIDING) | (colliding ? RP3DG_LF_WAS_COLLIDING : 0);
    }
    uint32_t nb = a.nb_contacts[i];
    if (nb > a.max_contacts) nb = a.max_contacts;
    uint32_t idx[MAX_RAW];
    v3 lp1[MAX_RAW];
    for (uint32_t k = 0; k < nb; k++) {
        idx[k] = k;
        const float4 l = a.local1[size_t(k) * a.n + i];
        lp1[k] = V(l.x, l.y, l.z);
    }
    if (nb > 0 && colliding) {
        if (nb > 4) {
            const float4 nd = a.normal_depth[i];
            const float4 q = a.rot1[i];
            uint32_t cand[MAX_RAW];
            reduce_points(idx, nb, LocalPoints{lp1}, V(nd.x, nd.y, nd.z), Q(q.x, q.y, q.z, q.w), cand);
        }
        remove_duplicates(idx, nb, LocalPoints{lp1});
    }
    const uint32_t m = nb < 4 ? nb : 4;
    float4 nd[4], l1[4], l2[4];
    for (uint32_t k = 0; k < m; k++) {
        const size_t o = size_t(idx[k]) * a.n + i;
        nd[k] = a.normal_depth[o]; l1[k] = a.local1[o]; l2[k] = a.local2[o];
    }
    for (uint32_t k = 0; k < m; k++) {
        const size_t o = size_t(k) * a.n + i;
        a.normal_depth[o] = nd[k]; a.local1[o] = l1[k]; a.local2[o] = l2[k];
    }
    if (a.kept) {
        uchar4 kk;
        kk.x = uint8_t(0 < m ? idx[0] : 255u); kk.y = uint8_t(1 < m ? idx[1] : 255u);
        kk.z = uint8_t(2 < m ? idx[2] : 255u); kk.w = uint8_t(3 < m ? idx[3] : 255u);
        reinterpret_cast<uchar4*>(a.kept)[i] = kk;
    }
    a.nb_contacts[i] = uint8_t(m);
}

cudaError_t launch_contacts_reduce(const ReduceArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    contacts_reduce_kernel<<<(a.n + 127) / 128, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace rp3dg
