// Debug rendering of a world as headless device buffers: the lines and
// triangles DebugRenderer builds (src/utils/DebugRenderer.cpp:62-545) for
// every collider (world AABB, broad-phase fat AABB, collision shape, face
// normals) and every contact point (a small sphere and the normal), with the
// reference's vertex expressions, primitive order and colours.  One CTA per
// collider; the host gives each collider its output offsets, the contact
// primitives come first (DebugRenderer::onContact runs during the update,
// computeDebugRenderingPrimitives at its end).
#include <cuda_runtime.h>

#include <cmath>

#include "debug_launch.h"
#include "rp3dg_math.cuh"
#include "shape_aabb.cuh"

namespace rp3dg {

// DebugRenderer's default colours (DebugRenderer.cpp:48-53, DebugColor)
constexpr uint32_t COLOR_AABB = 0xff00ffu, COLOR_BP_AABB = 0xffff00u, COLOR_SHAPE = 0x00ff00u,
                   COLOR_CONTACT_POINT = 0xff0000u, COLOR_CONTACT_NORMAL = 0xffffffu, COLOR_SHAPE_NORMAL = 0x0000ffu;

void make_debug_trig(DebugTrig* t) {
    // drawSphere / drawCapsule (DebugRenderer.cpp:146-297): float angles
    const float pi = 3.141592653589f;   // PI_RP3D (configuration.h:123)
    const float sectorStep = 2 * pi / DEBUG_SECTORS;
    const float stackStep = pi / DEBUG_STACKS;
    for (uint32_t i = 0; i <= uint32_t(DEBUG_STACKS); i++) {
        const float stackAngle = pi / 2 - i * stackStep;
        t->stack_cos[i] = std::cos(stackAngle);
        t->stack_sin[i] = std::sin(stackAngle);
    }
    for (uint32_t j = 0; j <= uint32_t(DEBUG_SECTORS); j++) {
        const float sectorAngle = j * sectorStep;
        t->sector_cos[j] = std::cos(sectorAngle);
        t->sector_sin[j] = std::sin(sectorAngle);
    }
}

void debug_collider_counts(uint32_t items, int kind, const uint32_t* face_counts, uint32_t nfaces, uint32_t hf_cols,
                           uint32_t hf_rows, uint32_t cm_vertices, uint32_t cm_triangles, uint32_t* lines,
                           uint32_t* tris) {
    uint32_t l = 0, t = 0;
    if (items & RP3DG_DEBUG_COLLIDER_AABB) l += 12;
    if (items & RP3DG_DEBUG_COLLIDER_BROADPHASE_AABB) l += 12;
    const bool shape = (items & RP3DG_DEBUG_COLLISION_SHAPE) != 0, normal = (items & RP3DG_DEBUG_COLLISION_SHAPE_NORMAL) != 0;
    if (shape || normal) {
        switch (kind) {
            case RP3DG_SHAPE_BOX:
                if (shape) t += 12;
                if (normal) l += 6;
                break;
            // drawSphere and drawCapsule add their triangles whenever they are called
            case RP3DG_SHAPE_SPHERE: t += DEBUG_SPHERE_TRIS; break;
            case RP3DG_SHAPE_CAPSULE: t += 360; break;
            case RP3DG_SHAPE_CONVEX_MESH:
                for (uint32_t f = 0; f < nfaces; f++)
                    if (shape && face_counts[f] >= 3) t += face_counts[f] - 2;
                if (normal) l += nfaces;
                break;
            case RP3DG_SHAPE_CONCAVE_MESH:
                if (shape) t += cm_triangles;
                if (normal) l += cm_vertices;
                break;
            case RP3DG_SHAPE_HEIGHTFIELD: {
                const uint32_t cells = (hf_cols > 1 && hf_rows > 1) ? (hf_cols - 1) * (hf_rows - 1) : 0u;
                if (shape) t += 2 * cells;
                if (normal) l += 4 * cells;
                break;
            }
            default: break;
        }
    }
    *lines = l;
    *tris = t;
}

namespace {

RD void put_line(rp3dg_debug_line* o, v3 a, v3 b, uint32_t c) {
    o->p1[0] = a.x; o->p1[1] = a.y; o->p1[2] = a.z; o->color1 = c;
    o->p2[0] = b.x; o->p2[1] = b.y; o->p2[2] = b.z; o->color2 = c;
}
RD void put_tri(rp3dg_debug_triangle* o, v3 a, v3 b, v3 c, uint32_t col) {
    o->p1[0] = a.x; o->p1[1] = a.y; o->p1[2] = a.z; o->color1 = col;
    o->p2[0] = b.x; o->p2[1] = b.y; o->p2[2] = b.z; o->color2 = col;
    o->p3[0] = c.x; o->p3[1] = c.y; o->p3[2] = c.z; o->color3 = col;
}

// drawAABB (DebugRenderer.cpp:69-91): line k of the 12
RD void aabb_line(v3 mn, v3 mx, int k, v3& a, v3& b) {
    switch (k) {
        case 0: a = V(mn.x, mn.y, mx.z); b = V(mx.x, mn.y, mx.z); break;
        case 1: a = V(mx.x, mn.y, mx.z); b = V(mx.x, mn.y, mn.z); break;
        case 2: a = V(mx.x, mn.y, mn.z); b = V(mn.x, mn.y, mn.z); break;
        case 3: a = V(mn.x, mn.y, mn.z); b = V(mn.x, mn.y, mx.z); break;
        case 4: a = V(mn.x, mx.y, mx.z); b = V(mx.x, mx.y, mx.z); break;
        case 5: a = V(mx.x, mx.y, mx.z); b = V(mx.x, mx.y, mn.z); break;
        case 6: a = V(mx.x, mx.y, mn.z); b = V(mn.x, mx.y, mn.z); break;
        case 7: a = V(mn.x, mx.y, mn.z); b = V(mn.x, mx.y, mx.z); break;
        case 8: a = V(mn.x, mn.y, mx.z); b = V(mn.x, mx.y, mx.z); break;
        case 9: a = V(mx.x, mn.y, mx.z); b = V(mx.x, mx.y, mx.z); break;
        case 10: a = V(mx.x, mn.y, mn.z); b = V(mx.x, mx.y, mn.z); break;
        default: a = V(mn.x, mn.y, mn.z); b = V(mn.x, mx.y, mn.z); break;
    }
}

// drawSphere vertex (i, j) (DebugRenderer.cpp:153-163)
RD v3 sphere_vertex(const DebugTrig& t, v3 pos, float r, uint32_t i, uint32_t j) {
    const float rc = r * t.stack_cos[i];
    const float z = r * t.stack_sin[i];
    const float x = rc * t.sector_cos[j];
    const float y = rc * t.sector_sin[j];
    return vadd(pos, V(x, y, z));
}
// triangle k of drawSphere (:165-181): stack 0 and the last stack have one
// triangle per sector, the others two
RD void sphere_tri(const DebugTrig& t, v3 pos, float r, uint32_t k, v3& a, v3& b, v3& c) {
    constexpr uint32_t S = DEBUG_SECTORS, W = DEBUG_SECTORS + 1;
    uint32_t i, j;
    bool first;
    if (k < S) { i = 0; j = k; first = false; }
    else if (k >= S + 2 * S * (DEBUG_STACKS - 2)) { i = DEBUG_STACKS - 1; j = k - (S + 2 * S * (DEBUG_STACKS - 2)); first = true; }
    else {
        const uint32_t q = k - S;
        i = 1 + q / (2 * S);
        j = (q % (2 * S)) / 2;
        first = (q & 1u) == 0;
    }
    const uint32_t a1 = i * W + j, a2 = a1 + W;
    auto vx = [&](uint32_t idx) { return sphere_vertex(t, pos, r, idx / W, idx % W); };
    if (first) { a = vx(a1); b = vx(a2); c = vx(a1 + 1); }
    else { a = vx(a1 + 1); b = vx(a2); c = vx(a2 + 1); }
}

// drawCapsule vertex of index idx (DebugRenderer.cpp:203-244): the upper
// half's 6 rings, then the lower half's 6
RD v3 capsule_vertex(const DebugTrig& t, const xform& T, float r, float halfHeight, uint32_t idx) {
    constexpr uint32_t W = DEBUG_SECTORS + 1, HALF = DEBUG_STACKS / 2;
    const bool upper = idx < (HALF + 1) * W;
    const uint32_t local = upper ? idx : idx - (HALF + 1) * W;
    const uint32_t i = local / W, j = local % W;
    const uint32_t st = upper ? i : HALF + i;
    const float rc = r * t.stack_cos[st];
    const float y = r * t.stack_sin[st];
    const float x = rc * t.sector_sin[j];
    const float z = rc * t.sector_cos[j];
    return xapply(T, V(x, upper ? y + halfHeight : y - halfHeight, z));
}
// triangle k of drawCapsule (:246-295)
RD void capsule_tri(const DebugTrig& t, const xform& T, float r, float hh, uint32_t k, v3& a, v3& b, v3& c) {
    constexpr uint32_t S = DEBUG_SECTORS, W = DEBUG_SECTORS + 1, HALF = DEBUG_STACKS / 2;
    uint32_t a1, a2;
    bool first;
    const uint32_t upper_n = S + 2 * S * (HALF - 1);   // 162
    const uint32_t lower_n = 2 * S * (HALF - 1) + S;   // 162
    if (k < upper_n) {
        uint32_t i, j;
        if (k < S) { i = 0; j = k; first = false; }
        else { const uint32_t q = k - S; i = 1 + q / (2 * S); j = (q % (2 * S)) / 2; first = (q & 1u) == 0; }
        a1 = i * W + j;
        a2 = a1 + W;
    } else if (k < upper_n + lower_n) {
        const uint32_t q = k - upper_n;
        uint32_t i, j;
        if (q < 2 * S * (HALF - 1)) { i = q / (2 * S); j = (q % (2 * S)) / 2; first = (q & 1u) == 0; }
        else { i = HALF - 1; j = q - 2 * S * (HALF - 1); first = true; }
        a1 = (HALF + 1) * W + i * W + j;
        a2 = a1 + W;
    } else {
        // the band between the two halves: per sector the second triangle first
        const uint32_t q = k - upper_n - lower_n;
        const uint32_t j = q / 2;
        first = (q & 1u) != 0;
        a1 = HALF * W + j;
        a2 = a1 + W;
    }
    if (first) { a = capsule_vertex(t, T, r, hh, a1); b = capsule_vertex(t, T, r, hh, a2); c = capsule_vertex(t, T, r, hh, a1 + 1); }
    else { a = capsule_vertex(t, T, r, hh, a1 + 1); b = capsule_vertex(t, T, r, hh, a2); c = capsule_vertex(t, T, r, hh, a2 + 1); }
}

// BoxShape::getVertexPosition (BoxShape.h:192-208)
RD v3 box_vertex(v3 he, uint32_t v) {
    return V(((0x66u >> v) & 1u) ? he.x : -he.x, ((0xCCu >> v) & 1u) ? he.y : -he.y, ((0x0Fu >> v) & 1u) ? he.z : -he.z);
}
// BoxShape::getFaceNormal (BoxShape.h:211-225)
RD v3 box_normal(uint32_t f) {
    switch (f) {
        case 0: return V(0.0f, 0.0f, 1.0f);
        case 1: return V(1.0f, 0.0f, 0.0f);
        case 2: return V(0.0f, 0.0f, -1.0f);
        case 3: return V(-1.0f, 0.0f, 0.0f);
        case 4: return V(0.0f, -1.0f, 0.0f);
        default: return V(0.0f, 1.0f, 0.0f);
    }
}
// the box's faces (PhysicsCommon::initBoxShapeHalfEdgeStructure)
__constant__ uint8_t c_box_faces[6][4] = {{0, 1, 2, 3}, {1, 5, 6, 2}, {4, 7, 6, 5}, {4, 0, 3, 7}, {4, 5, 1, 0}, {2, 6, 7, 3}};
// drawBox's triangles (DebugRenderer.cpp:112-124), over the transformed
// vertices 0..7 of its own numbering
__constant__ uint8_t c_box_tris[12][3] = {{0, 1, 5}, {0, 5, 4}, {1, 2, 6}, {1, 6, 5}, {2, 3, 6}, {3, 7, 6},
                                          {0, 7, 3}, {0, 4, 7}, {0, 2, 1}, {0, 3, 2}, {5, 6, 4}, {4, 6, 7}};
// drawBox's vertices (:101-108): signs of (x, y, z) times the half-extents
RD v3 draw_box_vertex(v3 he, uint32_t v) {
    const float sx = (v == 1 || v == 2 || v == 5 || v == 6) ? 1.0f : -1.0f;
    const float sy = v >= 4 ? 1.0f : -1.0f;
    const float sz = (v == 0 || v == 1 || v == 4 || v == 5) ? 1.0f : -1.0f;
    return V(sx > 0 ? he.x : -he.x, sy > 0 ? he.y : -he.y, sz > 0 ? he.z : -he.z);
}

RD v3 hf_vertex_dbg(const HfDesc& h, uint32_t x, uint32_t y) {
    const float height = h.heights[size_t(y) * h.ncol + x];
    const v3 v = V(-h.width * 0.5f + float(x), h.origin + height, -h.length * 0.5f + float(y));
    return V(v.x * h.scale[0], v.y * h.scale[1], v.z * h.scale[2]);
}

__global__ void __launch_bounds__(128) debug_colliders(const DebugArgs a) {
    const DebugJob J = a.jobs[blockIdx.x];
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    const rp3dg_shape sh = a.shapes[J.shape];
    const float4 p4 = a.wpos[J.row], q4 = a.wori[J.row];
    const xform T = X(V(p4.x, p4.y, p4.z), Q(q4.x, q4.y, q4.z, q4.w));
    uint32_t line = J.line;
    // Collider::getWorldAABB: computeTransformedAABB of the current transform
    if (a.items & RP3DG_DEBUG_COLLIDER_AABB) {
        if (tid < 12) {
            v3 mn, mx, p, q;
            shape_transformed_aabb(sh.kind, sh.params[0], a.bounds[2 * J.shape], a.bounds[2 * J.shape + 1], T, mn, mx);
            aabb_line(mn, mx, int(tid), p, q);
            put_line(a.lines + line + tid, p, q, COLOR_AABB);
        }
        line += 12;
    }
    if (a.items & RP3DG_DEBUG_COLLIDER_BROADPHASE_AABB) {
        if (tid < 12) {
            const float4 fn = a.fmin[J.row], fx = a.fmax[J.row];
            v3 p, q;
            aabb_line(V(fn.x, fn.y, fn.z), V(fx.x, fx.y, fx.z), int(tid), p, q);
            put_line(a.lines + line + tid, p, q, COLOR_BP_AABB);
        }
        line += 12;
    }
    const bool shape = (a.items & RP3DG_DEBUG_COLLISION_SHAPE) != 0;
    const bool normal = (a.items & RP3DG_DEBUG_COLLISION_SHAPE_NORMAL) != 0;
    if (!shape && !normal) return;
    switch (sh.kind) {
        case RP3DG_SHAPE_BOX: {
            const v3 he = V(sh.params[0], sh.params[1], sh.params[2]);
            if (shape && tid < 12) {
                const uint8_t* k = c_box_tris[tid];
                put_tri(a.tris + J.tri + tid, xapply(T, draw_box_vertex(he, k[0])), xapply(T, draw_box_vertex(he, k[1])),
                        xapply(T, draw_box_vertex(he, k[2])), COLOR_SHAPE);
            }
            if (normal && tid < 6) {
                const uint8_t* f = c_box_faces[tid];
                const v3 s = vadd(vadd(vadd(box_vertex(he, f[0]), box_vertex(he, f[1])), box_vertex(he, f[2])), box_vertex(he, f[3]));
                const v3 facePoint = V(0.25f * s.x, 0.25f * s.y, 0.25f * s.z);
                const v3 n = box_normal(tid);
                const v3 normalPoint = vadd(facePoint, V(1.0f * n.x, 1.0f * n.y, 1.0f * n.z));
                put_line(a.lines + line + tid, xapply(T, facePoint), xapply(T, normalPoint), COLOR_SHAPE_NORMAL);
            }
            break;
        }
        case RP3DG_SHAPE_SPHERE:
            for (uint32_t k = tid; k < DEBUG_SPHERE_TRIS; k += nt) {
                v3 p, q, r;
                sphere_tri(a.trig, T.p, sh.params[0], k, p, q, r);
                put_tri(a.tris + J.tri + k, p, q, r, COLOR_SHAPE);
            }
            break;
        case RP3DG_SHAPE_CAPSULE: {
            const float height = sh.params[1] + sh.params[1];
            const float halfHeight = 0.5f * height;
            for (uint32_t k = tid; k < 360; k += nt) {
                v3 p, q, r;
                capsule_tri(a.trig, T, sh.params[0], halfHeight, k, p, q, r);
                put_tri(a.tris + J.tri + k, p, q, r, COLOR_SHAPE);
            }
            break;
        }
        case RP3DG_SHAPE_CONVEX_MESH: {
            // drawConvexMesh (:299-347): per face, triangles of consecutive
            // vertex triples, then the face normal from the centroid of the
            // transformed vertices
            if (tid != 0) break;
            const MeshHdr* h = reinterpret_cast<const MeshHdr*>(a.mesh_words) + sh.mesh;
            const uint32_t* w = a.mesh_words;
            auto vtx = [&](uint32_t v) {
                const uint32_t o = h->off_sverts + 3 * v;
                return V(__uint_as_float(w[o]), __uint_as_float(w[o + 1]), __uint_as_float(w[o + 2]));
            };
            uint32_t tri = J.tri;
            for (uint32_t f = 0; f < h->nf; f++) {
                const uint32_t fs = w[h->off_face_start + f], fc = w[h->off_face_count + f];
                v3 centroid = V(0.0f, 0.0f, 0.0f);
                for (uint32_t v = 2; v < fc; v++) {
                    const v3 v1 = xapply(T, vtx(w[h->off_face_verts + fs + v - 2]));
                    const v3 v2 = xapply(T, vtx(w[h->off_face_verts + fs + v - 1]));
                    const v3 v3_ = xapply(T, vtx(w[h->off_face_verts + fs + v]));
                    if (v == 2) centroid = vadd(centroid, vadd(v1, v2));
                    centroid = vadd(centroid, v3_);
                    if (shape) put_tri(a.tris + tri++, v1, v2, v3_, COLOR_SHAPE);
                }
                if (normal) {
                    const float nfv = float(fc);
                    centroid = V(centroid.x / nfv, centroid.y / nfv, centroid.z / nfv);
                    const uint32_t o = h->off_normals + 3 * f;
                    const v3 fn = qrot(T.q, V(__uint_as_float(w[o]), __uint_as_float(w[o + 1]), __uint_as_float(w[o + 2])));
                    const v3 normalPoint = vadd(centroid, V(fn.x * 1.0f, fn.y * 1.0f, fn.z * 1.0f));
                    put_line(a.lines + line++, centroid, normalPoint, COLOR_SHAPE_NORMAL);
                }
            }
            break;
        }
        case RP3DG_SHAPE_CONCAVE_MESH: {
            // drawConcaveMeshShape (:350-383): every triangle (scaled vertices),
            // then a normal line per vertex
            const CmDesc cm = a.cm[sh.mesh];
            auto ld = [](const float* p, uint32_t v) { return V(p[3 * v], p[3 * v + 1], p[3 * v + 2]); };
            if (shape)
                for (uint32_t k = tid; k < cm.nt; k += nt) {
                    const v3 p0 = xapply(T, ld(cm.sverts, cm.tris[3 * k]));
                    const v3 p1 = xapply(T, ld(cm.sverts, cm.tris[3 * k + 1]));
                    const v3 p2 = xapply(T, ld(cm.sverts, cm.tris[3 * k + 2]));
                    put_tri(a.tris + J.tri + k, p0, p1, p2, COLOR_SHAPE);
                }
            if (normal)
                for (uint32_t v = tid; v < cm.nv; v += nt) {
                    const v3 vertex = xapply(T, ld(cm.sverts, v));
                    const v3 n = qrot(T.q, ld(cm.snormals, v));
                    put_line(a.lines + line + v, vertex, vadd(vertex, V(n.x * 1.0f, n.y * 1.0f, n.z * 1.0f)), COLOR_SHAPE_NORMAL);
                }
            break;
        }
        case RP3DG_SHAPE_HEIGHTFIELD: {
            // drawHeightFieldShape (:385-429): columns outer, rows inner
            const HfDesc h = a.hf[sh.mesh];
            if (h.ncol < 2 || h.nrow < 2) break;
            const uint32_t cells = (h.ncol - 1) * (h.nrow - 1);
            for (uint32_t c = tid; c < cells; c += nt) {
                const uint32_t i = c / (h.nrow - 1), j = c % (h.nrow - 1);
                const v3 p1 = xapply(T, hf_vertex_dbg(h, i, j));
                const v3 p2 = xapply(T, hf_vertex_dbg(h, i, j + 1));
                const v3 p3 = xapply(T, hf_vertex_dbg(h, i + 1, j));
                const v3 p4 = xapply(T, hf_vertex_dbg(h, i + 1, j + 1));
                if (shape) {
                    put_tri(a.tris + J.tri + 2 * c, p1, p2, p3, COLOR_SHAPE);
                    put_tri(a.tris + J.tri + 2 * c + 1, p3, p2, p4, COLOR_SHAPE);
                }
                if (normal) {
                    const v3 n = vunit(vcross(vsub(p2, p1), vsub(p3, p1)));
                    const v3 d = V(n.x * 1.0f, n.y * 1.0f, n.z * 1.0f);
                    put_line(a.lines + line + 4 * c, p1, vadd(p1, d), COLOR_SHAPE_NORMAL);
                    put_line(a.lines + line + 4 * c + 1, p2, vadd(p2, d), COLOR_SHAPE_NORMAL);
                    put_line(a.lines + line + 4 * c + 2, p3, vadd(p3, d), COLOR_SHAPE_NORMAL);
                    put_line(a.lines + line + 4 * c + 3, p4, vadd(p4, d), COLOR_SHAPE_NORMAL);
                }
            }
            break;
        }
        default: break;
    }
}

// DebugRenderer::onContact (:530-545): per contact point of the step a sphere
// of radius 0.1 at collider 1's local-to-world transform times the local
// point on collider 1, and the normal, 1 m long.
__global__ void __launch_bounds__(128) debug_contacts(const DebugArgs a) {
    const uint32_t k = blockIdx.x;
    if (k >= a.n_points) return;
    const int4 pt = a.points[k];
    const float4 p4 = a.snap_wpos[pt.x], q4 = a.snap_wori[pt.x];
    const xform T = X(V(p4.x, p4.y, p4.z), Q(q4.x, q4.y, q4.z, q4.w));
    const float4 l = a.l1[pt.y], nd = a.nd[pt.y];
    const v3 point = xapply(T, V(l.x, l.y, l.z));
    const bool spheres = (a.items & RP3DG_DEBUG_CONTACT_POINT) != 0;
    if (spheres)
        for (uint32_t t = threadIdx.x; t < DEBUG_SPHERE_TRIS; t += blockDim.x) {
            v3 p, q, r;
            sphere_tri(a.trig, point, 0.1f, t, p, q, r);
            put_tri(a.tris + uint32_t(pt.w) + t, p, q, r, COLOR_CONTACT_POINT);
        }
    if ((a.items & RP3DG_DEBUG_CONTACT_NORMAL) && threadIdx.x == 0)
        put_line(a.lines + uint32_t(pt.z), point, vadd(point, V(nd.x * 1.0f, nd.y * 1.0f, nd.z * 1.0f)), COLOR_CONTACT_NORMAL);
}

}  // namespace

cudaError_t launch_debug(const DebugArgs& a, cudaStream_t s) {
    if (a.n_points && (a.items & (RP3DG_DEBUG_CONTACT_POINT | RP3DG_DEBUG_CONTACT_NORMAL)))
        debug_contacts<<<a.n_points, 128, 0, s>>>(a);
    if (a.n_jobs) debug_colliders<<<a.n_jobs, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace rp3dg
