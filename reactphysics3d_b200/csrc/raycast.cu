// Batched world raycast: one thread traces one ray as PhysicsWorld::raycast
// does (reference src/collision/broadphase/DynamicAABBTree.cpp:684-747,
// src/systems/BroadPhaseSystem.cpp:224-240, src/collision/RaycastInfo.cpp:34-49,
// src/collision/Collider.cpp:173-192): the broad-phase tree in its stack order
// with the ray clipped by each accepted hit, the category filter, the ray
// taken into the collider's local space, the shape's own raycast, the hit
// taken back to world space.  Float expression trees follow the reference's
// (no contraction: the library is built with --fmad=false).
#include <cfloat>

#include "raycast_launch.h"
#include "rp3dg_math.cuh"

namespace rp3dg {
namespace {

constexpr int RAY_STACK = 96;
constexpr int RAY_BLOCK = 128;
// Eight resident CTAs per SM (64 registers, a few spilled): the traversal is
// latency-bound, and doubling the resident warps over the unconstrained
// allocation (103 registers, 4 CTAs) took 1 M rays over the 100,000-body
// terrain from 25.1 to 20.3 ms with the same results.
#ifndef RAY_MIN_BLOCKS
#define RAY_MIN_BLOCKS 8
#endif

struct LocalHit {
    v3 point, normal;
    float fraction;
};

RD float comp(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
RD int iclamp(int v, int lo, int hi) {  // clamp(int, int, int): std::min(std::max(v, lo), hi)
    const int m = (v < lo) ? lo : v;
    return (hi < m) ? hi : m;
}

// AABB::testRayIntersect (AABB.h:285-314)
RD bool ray_aabb(float4 lo, float4 hi, v3 o, v3 inv, float maxf) {
    float t1 = (lo.x - o.x) * inv.x;
    float t2 = (hi.x - o.x) * inv.x;
    float tmin = smin(t1, t2);
    float tmax = smax(t1, t2);
    tmax = smin(tmax, maxf);
    t1 = (lo.y - o.y) * inv.y;
    t2 = (hi.y - o.y) * inv.y;
    tmin = smax(tmin, smin(t1, t2));
    tmax = smin(tmax, smax(t1, t2));
    t1 = (lo.z - o.z) * inv.z;
    t2 = (hi.z - o.z) * inv.z;
    tmin = smax(tmin, smin(t1, t2));
    tmax = smin(tmax, smax(t1, t2));
    return tmax >= smax(tmin, 0.0f);
}

// SphereShape::raycast (SphereShape.cpp:61-104) and
// CapsuleShape::raycastWithSphereEndCap (CapsuleShape.cpp:243-286): the
// sphere of radius r centred at c.
RD bool ray_sphere_at(v3 p1, v3 p2, v3 c, float maxf, float r, v3& point, float& fraction) {
    const v3 m = vsub(p1, c);
    const float cc = vdot(m, m) - r * r;
    if (cc < 0.0f) return false;
    const v3 d = vsub(p2, p1);
    const float b = vdot(m, d);
    if (b > 0.0f) return false;
    const float len2 = vlen2(d);
    const float disc = b * b - len2 * cc;
    if (disc < 0.0f || len2 < MACHINE_EPSILON) return false;
    float t = -b - sqrtf(disc);
    if (t < maxf * len2) {
        t /= len2;
        fraction = t;
        point = vadd(p1, vmul(d, t));
        return true;
    }
    return false;
}

RD bool ray_sphere(v3 p1, v3 p2, float maxf, float r, LocalHit& h) {
    // the sphere's raycast uses the ray origin itself (m = point1)
    const v3 m = p1;
    const float c = vdot(m, m) - r * r;
    if (c < 0.0f) return false;
    const v3 d = vsub(p2, p1);
    const float b = vdot(m, d);
    if (b > 0.0f) return false;
    const float len2 = vlen2(d);
    const float disc = b * b - len2 * c;
    if (disc < 0.0f || len2 < MACHINE_EPSILON) return false;
    float t = -b - sqrtf(disc);
    if (t < maxf * len2) {
        t /= len2;
        h.fraction = t;
        h.point = vadd(p1, vmul(d, t));
        h.normal = h.point;
        return true;
    }
    return false;
}

// CapsuleShape::raycast (CapsuleShape.cpp:97-240): segment p-q on the y axis
RD bool ray_capsule(v3 p1, v3 p2, float maxf, float r, float hh, LocalHit& h) {
    const v3 n = vsub(p2, p1);
    const float eps = 0.01f;
    const v3 p = V(0.0f, -hh, 0.0f), q = V(0.0f, hh, 0.0f);
    const v3 d = vsub(q, p);
    const v3 m = vsub(p1, p);
    const float mDotD = vdot(m, d), nDotD = vdot(n, d), dDotD = vdot(d, d);
    const float vec1DotD = vdot(vsub(p1, V(0.0f, -hh - r, 0.0f)), d);
    if (vec1DotD < 0.0f && vec1DotD + nDotD < 0.0f) return false;
    const float extra = 2.0f * r * d.y;
    if (vec1DotD > dDotD + extra && vec1DotD + nDotD > dDotD + extra) return false;
    const float nDotN = vdot(n, n), mDotN = vdot(m, n);
    const float a = dDotD * nDotN - nDotD * nDotD;
    const float k = vdot(m, m) - r * r;
    const float c = dDotD * k - mDotD * mDotD;
    auto cap = [&](v3 centre) -> bool {
        v3 hp;
        float hf;
        if (!ray_sphere_at(p1, p2, centre, maxf, r, hp, hf)) return false;
        h.fraction = hf;
        h.point = hp;
        h.normal = vsub(hp, centre);
        return true;
    };
    if (fabsf(a) < eps) {
        if (c > 0.0f) return false;
        if (mDotD < 0.0f) return cap(p);
        if (mDotD > dDotD) return cap(q);
        return false;
    }
    const float b = dDotD * mDotN - nDotD * mDotD;
    const float disc = b * b - a * c;
    if (disc < 0.0f) return false;
    const float t = (-b - sqrtf(disc)) / a;
    const float value = mDotD + t * nDotD;
    if (value < 0.0f) return cap(p);
    if (value > dDotD) return cap(q);
    if (t < 0.0f || t > maxf) return false;
    const v3 lp = vadd(p1, vmul(n, t));
    h.fraction = t;
    h.point = lp;
    const v3 v = vsub(lp, p);
    const v3 w = vmul(d, vdot(v, d) / vlen2(d));
    h.normal = vunit(vsub(lp, vadd(p, w)));
    return true;
}

// BoxShape::raycast (BoxShape.cpp:62-119): slabs, the entering face's
// (unnormalised) normal
RD bool ray_box(v3 p1, v3 p2, float maxf, v3 he, LocalHit& h) {
    const v3 d = vsub(p2, p1);
    float tmin = -FLT_MAX, tmax = FLT_MAX;
    v3 nd = V(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < 3; i++) {
        const float di = comp(d, i), pi = comp(p1, i), hi = comp(he, i);
        if (fabsf(di) < MACHINE_EPSILON) {
            if (pi > hi || pi < -hi) return false;
        } else {
            const float inv = 1.0f / di;
            float t1 = (-hi - pi) * inv;
            float t2 = (hi - pi) * inv;
            v3 cn = V(i == 0 ? -hi : 0.0f, i == 1 ? -hi : 0.0f, i == 2 ? -hi : 0.0f);
            if (t1 > t2) {
                const float tt = t1;
                t1 = t2;
                t2 = tt;
                cn = vneg(cn);
            }
            if (t1 > tmin) {
                tmin = t1;
                nd = cn;
            }
            tmax = smin(tmax, t2);
            if (tmin > maxf) return false;
            if (tmin > tmax) return false;
        }
    }
    if (tmin < 0.0f || tmin > maxf) return false;
    h.point = vadd(p1, vmul(d, tmin));
    h.fraction = tmin;
    h.normal = nd;
    return true;
}

// ConvexMeshShape::raycast (ConvexMeshShape.cpp:107-172): face planes from
// the scaled face normals and the mesh's (unscaled) first vertex of each face
RD bool ray_mesh(v3 p1, v3 p2, float maxf, const MeshHdr* H, const uint32_t* w, LocalHit& h) {
    const v3 d = vsub(p2, p1);
    float tmin = 0.0f, tmax = maxf;
    v3 cn = V(0.0f, 0.0f, 0.0f);
    bool found = false;
    const uint32_t nf = H->nf;
    for (uint32_t f = 0; f < nf; f++) {
        const uint32_t on = H->off_normals + 3 * f;
        const v3 nrm = V(__uint_as_float(w[on]), __uint_as_float(w[on + 1]), __uint_as_float(w[on + 2]));
        const uint32_t v0 = w[H->off_face_verts + w[H->off_face_start + f]];
        const uint32_t ov = H->off_verts + 3 * v0;
        const v3 fp = V(__uint_as_float(w[ov]), __uint_as_float(w[ov + 1]), __uint_as_float(w[ov + 2]));
        const float denom = vdot(nrm, d);
        const float planeD = vdot(nrm, fp);
        const float dist = planeD - vdot(nrm, p1);
        if (denom == 0.0f) {
            if (dist < 0.0f) return false;
        } else {
            const float t = dist / denom;
            if (denom < 0.0f) {
                if (t > tmin) {
                    tmin = t;
                    cn = nrm;
                    found = true;
                }
            } else {
                if (t < tmax) tmax = t;
            }
            if (tmin > tmax) return false;
        }
    }
    if (!found) return false;
    h.point = vadd(p1, vmul(d, tmin));
    h.fraction = tmin;
    h.normal = cn;
    return true;
}

// AABB::raycast (AABB.h:317-357)
RD bool aabb_raycast(v3 mn, v3 mx, v3 p1, v3 p2, v3& hit) {
    float tmin = 0.0f, tmax = FLT_MAX;
    const float eps = 0.00001f;
    const v3 d = vsub(p2, p1);
    for (int i = 0; i < 3; i++) {
        const float di = comp(d, i), pi = comp(p1, i), lo = comp(mn, i), hi = comp(mx, i);
        if (fabsf(di) < eps) {
            if (pi < lo || pi > hi) return false;
        } else {
            const float inv = 1.0f / di;
            float t1 = (lo - pi) * inv;
            float t2 = (hi - pi) * inv;
            if (t1 > t2) {
                const float tt = t2;
                t2 = t1;
                t1 = tt;
            }
            tmin = smax(tmin, t1);
            tmax = smin(tmax, t2);
            if (tmin > tmax) return false;
        }
    }
    hit = vadd(p1, vmul(d, tmin));
    return true;
}

// TriangleShape::raycast (TriangleShape.cpp:143-230), FRONT side (the
// ConcaveShape default the height field passes on)
RD bool ray_triangle(v3 p1, v3 p2, float maxf, v3 a, v3 b, v3 c, LocalHit& h) {
    const v3 pq = vsub(p2, p1);
    const v3 pa = vsub(a, p1), pb = vsub(b, p1), pc = vsub(c, p1);
    const v3 m = vcross(pq, pc);
    float u = vdot(pb, m);
    if (u < 0.0f) return false;
    float v = -vdot(pa, m);
    if (v < 0.0f) return false;
    float w = vdot(pa, vcross(pq, pb));
    if (w < 0.0f) return false;
    if (fabsf(u - 0.0f) < MACHINE_EPSILON && fabsf(v - 0.0f) < MACHINE_EPSILON && fabsf(w - 0.0f) < MACHINE_EPSILON)
        return false;
    const float denom = 1.0f / (u + v + w);
    u *= denom;
    v *= denom;
    w *= denom;
    const v3 lp = vadd(vadd(vmul(a, u), vmul(b, v)), vmul(c, w));
    const float hf = vdot(vsub(lp, p1), pq) / vlen2(pq);
    if (hf < 0.0f || hf > maxf) return false;
    v3 nrm = vnormalize(vcross(vsub(b, a), vsub(c, a)));
    nrm = vdot(nrm, pq) > 0.0f ? vneg(nrm) : nrm;
    h.point = lp;
    h.fraction = hf;
    h.normal = nrm;
    return true;
}

// HeightField::getVertexAt (HeightField.cpp:386-393)
RD v3 hf_vertex(const HfDesc& H, int x, int y) {
    const float height = H.heights[size_t(y) * H.ncol + size_t(x)];
    return V(-H.width * 0.5f + float(x), H.origin + height, -H.length * 0.5f + float(y));
}

// HeightField::raycast with computeEnteringRayGridCoordinates
// (HeightField.cpp:258-384) on the ray already in the field's unscaled
// space: a grid walk from the cell where the ray enters the bounds, both
// triangles of each cell tested against the unclipped ray, a later hit at an
// equal fraction replacing an earlier one.  The reference's walk does not end
// when the ray's z direction is exactly zero and it enters on a cell
// boundary; this walk stops after as many cells as the grid can cross
// (*limit set).
RD bool ray_heightfield(v3 p1, v3 p2, float maxf, const HfDesc& H, LocalHit& h, bool* limit) {
    const v3 mn = V(H.bmin[0], H.bmin[1], H.bmin[2]), mx = V(H.bmax[0], H.bmax[1], H.bmax[2]);
    v3 g;
    if (!aabb_raycast(mn, mx, p1, p2, g)) return false;
    const v3 ext = vsub(mx, mn);
    const int ni = int(H.ncol) - 1, nj = int(H.nrow) - 1;
    g = vsub(g, mn);
    const float stepI = ext.x / float(ni), stepJ = ext.z / float(nj);
    int i = iclamp(int(g.x / stepI), 0, ni - 1);
    int j = iclamp(int(g.z / stepJ), 0, nj - 1);
    const v3 d = vsub(p2, p1);
    const int si = d.x > 0.0f ? 1 : (d.x < 0.0f ? -1 : 0);
    const int sj = d.z > 0.0f ? 1 : (d.z < 0.0f ? -1 : 0);
    const float nextI = float(si >= 0 ? i + 1 : i), nextJ = float(sj >= 0 ? j + 1 : j);
    const float sizeI = ext.x / float(ni), sizeJ = ext.z / float(nj);
    float tMaxI = ((nextI * sizeI) - g.x) / d.x;
    float tMaxJ = ((nextJ * sizeJ) - g.z) / d.z;
    const float tDeltaI = sizeI / fabsf(d.x), tDeltaJ = sizeJ / fabsf(d.z);
    float smallest = maxf;
    bool hit = false;
    const int max_cells = ni + nj + 2;
    int cells = 0;
    while (i >= 0 && i < ni && j >= 0 && j < nj) {
        if (cells++ >= max_cells) {
            *limit = true;
            break;
        }
        const v3 q1 = hf_vertex(H, i, j), q2 = hf_vertex(H, i, j + 1);
        const v3 q3 = hf_vertex(H, i + 1, j), q4 = hf_vertex(H, i + 1, j + 1);
        LocalHit t;
        if (ray_triangle(p1, p2, maxf, q1, q2, q3, t) && t.fraction <= smallest) {
            h = t;
            smallest = t.fraction;
            hit = true;
        }
        if (ray_triangle(p1, p2, maxf, q3, q2, q4, t) && t.fraction <= smallest) {
            h = t;
            smallest = t.fraction;
            hit = true;
        }
        if (si == 0 && sj == 0) break;
        if (tMaxI < tMaxJ) {
            tMaxI += tDeltaI;
            i += si;
        } else {
            tMaxJ += tDeltaJ;
            j += sj;
        }
    }
    return hit;
}

// ConcaveMeshShape::raycast (ConcaveMeshShape.cpp:179-274): the ray without
// the mesh's scale walks the mesh's tree (DynamicAABBTree::raycast,
// DynamicAABBTree.cpp:684-747, whose callback collects every leaf it reaches
// and returns the ray's maxFraction, so the walk is never clipped), then each
// collected triangle, scaled, is tested in that order against the unscaled
// ray (TriangleShape::raycast, FRONT side), a hit at a fraction <= the
// smallest so far replacing the current one.
constexpr int MESH_RAY_STACK = 64;
__device__ __noinline__ bool ray_concave_mesh(v3 p1, v3 p2, float maxf, const CmDesc& cm, LocalHit& h, bool* overflow) {
    const v3 is = V(cm.inv_scale[0], cm.inv_scale[1], cm.inv_scale[2]);
    const v3 s1 = vcmul(p1, is), s2 = vcmul(p2, is);
    const v3 d = vsub(s2, s1);
    const v3 dinv = V(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float smallest = maxf;
    bool hit = false;
    int stack[MESH_RAY_STACK];
    int sp = 0;
    stack[sp++] = cm.root;
    while (sp > 0) {
        const int id = stack[--sp];
        if (id < 0) continue;
        const float4 lo = __ldg(&cm.nodes[id].lo), hi = __ldg(&cm.nodes[id].hi);
        if (!ray_aabb(lo, hi, s1, dinv, maxf)) continue;
        const int c0 = __float_as_int(lo.w);
        if (c0 <= -2) {
            const uint32_t tri = uint32_t(-2 - c0);
            const uint32_t i0 = __ldg(cm.tris + 3 * tri), i1 = __ldg(cm.tris + 3 * tri + 1), i2 = __ldg(cm.tris + 3 * tri + 2);
            auto ld = [&](uint32_t v) { return V(__ldg(cm.sverts + 3 * v), __ldg(cm.sverts + 3 * v + 1), __ldg(cm.sverts + 3 * v + 2)); };
            LocalHit th;
            if (ray_triangle(p1, p2, maxf, ld(i0), ld(i1), ld(i2), th) && th.fraction <= smallest) {
                h = th;
                smallest = th.fraction;
                hit = true;
            }
            // the callback's answer is the ray's maxFraction: 0 ends the walk
            if (maxf == 0.0f) break;
        } else {
            if (sp + 2 > MESH_RAY_STACK) {
                *overflow = true;
                break;
            }
            stack[sp++] = c0;
            stack[sp++] = __float_as_int(hi.w);
        }
    }
    return hit;
}

// Collider::raycast: the ray into the collider's local space
// (localToWorld.getInverse() * point), the shape's raycast, the hit point and
// the rotated, normalised normal back in world space.
RD bool collider_raycast(const RayArgs& a, int4 col, v3 p1, v3 p2, float maxf, LocalHit& h, int* flags) {
    const float4 tp = a.c_wpos[col.x], tq = a.c_wori[col.x];
    const quat q = Q(tq.x, tq.y, tq.z, tq.w);
    const quat iq = qinv(q);
    const v3 ip = qrot(iq, V(-tp.x, -tp.y, -tp.z));
    const v3 l1 = vadd(qrot(iq, p1), ip), l2 = vadd(qrot(iq, p2), ip);
    const rp3dg_shape s = a.shapes[col.z];
    bool hit = false;
    switch (s.kind) {
        case RP3DG_SHAPE_SPHERE: hit = ray_sphere(l1, l2, maxf, s.params[0], h); break;
        case RP3DG_SHAPE_CAPSULE: hit = ray_capsule(l1, l2, maxf, s.params[0], s.params[1], h); break;
        case RP3DG_SHAPE_BOX: hit = ray_box(l1, l2, maxf, V(s.params[0], s.params[1], s.params[2]), h); break;
        case RP3DG_SHAPE_CONVEX_MESH:
            hit = ray_mesh(l1, l2, maxf, reinterpret_cast<const MeshHdr*>(a.mesh_words) + s.mesh, a.mesh_words, h);
            break;
        case RP3DG_SHAPE_HEIGHTFIELD: {
            if (s.mesh < 0 || uint32_t(s.mesh) >= a.nb_hfields) break;
            const HfDesc H = a.hfields[s.mesh];
            // HeightFieldShape::raycast (HeightFieldShape.cpp:76-90)
            const v3 is = V(1.0f / H.scale[0], 1.0f / H.scale[1], 1.0f / H.scale[2]);
            bool limit = false;
            hit = ray_heightfield(vcmul(l1, is), vcmul(l2, is), maxf, H, h, &limit);
            if (hit) h.point = vcmul(h.point, V(H.scale[0], H.scale[1], H.scale[2]));
            if (limit) *flags |= 1;
            break;
        }
        case RP3DG_SHAPE_CONCAVE_MESH: {
            if (s.mesh < 0 || uint32_t(s.mesh) >= a.nb_cmeshes) break;
            bool overflow = false;
            hit = ray_concave_mesh(l1, l2, maxf, a.cmeshes[s.mesh], h, &overflow);
            if (overflow) atomicOr(a.error, 1u);
            break;
        }
        default: break;
    }
    if (!hit) return false;
    h.point = vadd(qrot(q, h.point), V(tp.x, tp.y, tp.z));
    h.normal = vnormalize(qrot(q, h.normal));
    return true;
}

__global__ void __launch_bounds__(RAY_BLOCK, RAY_MIN_BLOCKS) world_raycast_kernel(const RayArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const rp3dg_ray R = a.rays[i];
    const v3 p1 = V(R.point1[0], R.point1[1], R.point1[2]), p2 = V(R.point2[0], R.point2[1], R.point2[2]);
    float maxf = R.max_fraction;
    const v3 dir = vsub(p2, p1);
    const v3 inv = V(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
    rp3dg_raycast_hit* out = a.hits + size_t(i) * a.max_hits;
    uint32_t count = 0;
    int stack[RAY_STACK];
    int sp = 0;
    stack[sp++] = a.root;
    while (sp > 0) {
        const int id = stack[--sp];
        if (id < 0) continue;
        const RayNode nd = a.nodes[id];
        if (!ray_aabb(nd.lo, nd.hi, p1, inv, maxf)) continue;
        const int c0 = __float_as_int(nd.lo.w);
        if (c0 <= -2) {
            const int c = -2 - c0;
            const int4 col = a.colliders[c];
            float ret = -1.0f;
            if ((R.category_mask & uint32_t(col.w)) != 0u) {
                LocalHit h;
                int flags = 0;
                if (collider_raycast(a, col, p1, p2, maxf, h, &flags)) {
                    rp3dg_raycast_hit rec;
                    rec.world_point[0] = h.point.x; rec.world_point[1] = h.point.y; rec.world_point[2] = h.point.z;
                    rec.world_normal[0] = h.normal.x; rec.world_normal[1] = h.normal.y; rec.world_normal[2] = h.normal.z;
                    rec.hit_fraction = h.fraction;
                    rec.body = col.y;
                    rec.collider = c;
                    rec.flags = flags;
                    if (a.mode == RP3DG_RAYCAST_ALL) {
                        if (count < a.max_hits) out[count] = rec;
                        ret = 1.0f;
                    } else {
                        if (a.max_hits) out[0] = rec;
                        ret = (a.mode == RP3DG_RAYCAST_ANY) ? 0.0f : h.fraction;
                    }
                    count++;
                } else {
                    ret = maxf;  // RaycastTest::raycastAgainstShape without a hit
                }
            }
            if (ret == 0.0f) break;
            if (ret > 0.0f && ret < maxf) maxf = ret;
        } else {
            if (sp + 2 > RAY_STACK) {
                atomicOr(a.error, 1u);
                break;
            }
            stack[sp++] = c0;
            stack[sp++] = __float_as_int(nd.hi.w);
        }
    }
    a.nb_hits[i] = count;
}

}  // namespace

cudaError_t launch_world_raycast(const RayArgs& a, cudaStream_t stream) {
    if (a.n == 0) return cudaSuccess;
    world_raycast_kernel<<<(a.n + RAY_BLOCK - 1) / RAY_BLOCK, RAY_BLOCK, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace rp3dg
