/* Test infrastructure, not product code: a plain-C restatement of
 * ReactPhysics3D v0.10.2's narrow phase (single precision), used only as a
 * checker.  Every function cites the reference file:line it restates; the
 * operation order of every floating-point expression is the reference's, so
 * that, compiled without contraction (-ffp-contract=off) on an x86-64 SSE
 * target, results are bit-identical to the reference's float build.
 * All paths below are inside the reference project.
 */
#include "rp3d_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* constants (configuration.h:114-120, GJKAlgorithm.h:44-46,          */
/* SATAlgorithm.cpp:43-44, VoronoiSimplex.cpp:33)                     */
/* ------------------------------------------------------------------ */
#define MACHINE_EPSILON FLT_EPSILON
#define DECIMAL_LARGEST FLT_MAX
#define DECIMAL_SMALLEST (-FLT_MAX)
static const float REL_ERROR = 1.0e-3f;
#define REL_ERROR_SQUARE (REL_ERROR * REL_ERROR)
static const float SAT_REL_TOL = 1.002f;
static const float SAT_ABS_TOL = 0.0005f;
static const float SIMPLEX_EPS = 0.0001f;
#define MAX_CONTACTS RP3DG_MAX_CONTACTS_PER_PAIR

/* ------------------------------------------------------------------ */
/* math (Vector3.h, Vector3.cpp, Quaternion.h, Transform.h,           */
/* mathematics_functions.h)                                           */
/* ------------------------------------------------------------------ */
typedef struct { float x, y, z; } v3;
typedef struct { float x, y, z, w; } quat;
typedef struct { v3 p; quat q; } xform;

static v3 V(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
/* operator*(Vector3, decimal) = Vector3(number * v.x, ...) (Vector3.h:322-324) */
static v3 vmul(v3 a, float s) { return V(s * a.x, s * a.y, s * a.z); }
static v3 vdivs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static v3 vcmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 vcross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static float vlen2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static float vlen(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
/* Vector3::getUnit (Vector3.cpp:33-43) */
static v3 vunit(v3 a) {
    float l = vlen(a);
    if (l < MACHINE_EPSILON) return a;
    float inv = 1.0f / l;
    return V(a.x * inv, a.y * inv, a.z * inv);
}
/* Vector3::normalize (Vector3.h:219-227) */
static v3 vnormalize(v3 a) {
    float l = vlen(a);
    if (l < MACHINE_EPSILON) return a;
    return V(a.x / l, a.y / l, a.z / l);
}
static float fmin_std(float a, float b) { return (b < a) ? b : a; } /* std::min */
static float fmax_std(float a, float b) { return (a < b) ? b : a; } /* std::max */
static float clampf_std(float v, float lo, float hi) { return fmin_std(fmax_std(v, lo), hi); }

static quat Q(float x, float y, float z, float w) { quat r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }
static quat qinv(quat q) { return Q(-q.x, -q.y, -q.z, q.w); } /* Quaternion.h:283-287 */
/* Quaternion * Quaternion (Quaternion.h:346-359) */
static quat qmul(quat a, quat b) {
    return Q(a.w * b.x + b.w * a.x + a.y * b.z - a.z * b.y,
             a.w * b.y + b.w * a.y + a.z * b.x - a.x * b.z,
             a.w * b.z + b.w * a.z + a.x * b.y - a.y * b.x,
             a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
/* Quaternion * Vector3 (Quaternion.h:363-379) */
static v3 qrot(quat q, v3 p) {
    const float prodX = q.w * p.x + q.y * p.z - q.z * p.y;
    const float prodY = q.w * p.y + q.z * p.x - q.x * p.z;
    const float prodZ = q.w * p.z + q.x * p.y - q.y * p.x;
    const float prodW = -q.x * p.x - q.y * p.y - q.z * p.z;
    return V(q.w * prodX - prodY * q.z + prodZ * q.y - prodW * q.x,
             q.w * prodY - prodZ * q.x + prodX * q.z - prodW * q.y,
             q.w * prodZ - prodX * q.y + prodY * q.x - prodW * q.z);
}
static xform X(v3 p, quat q) { xform t; t.p = p; t.q = q; return t; }
/* Transform::getInverse (Transform.h:162-165) */
static xform xinv(xform t) { quat iq = qinv(t.q); return X(qrot(iq, vneg(t.p)), iq); }
/* Transform * Vector3 (Transform.h:193-195) */
static v3 xapply(xform t, v3 v) { return vadd(qrot(t.q, v), t.p); }
/* Transform * Transform (Transform.h:198-225) */
static xform xmul(xform a, xform b) {
    const quat o = a.q;
    const v3 p = b.p;
    const float prodX = o.w * p.x + o.y * p.z - o.z * p.y;
    const float prodY = o.w * p.y + o.z * p.x - o.x * p.z;
    const float prodZ = o.w * p.z + o.x * p.y - o.y * p.x;
    const float prodW = -o.x * p.x - o.y * p.y - o.z * p.z;
    v3 np = V(a.p.x + o.w * prodX - prodY * o.z + prodZ * o.y - prodW * o.x,
              a.p.y + o.w * prodY - prodZ * o.x + prodX * o.z - prodW * o.y,
              a.p.z + o.w * prodZ - prodX * o.y + prodY * o.x - prodW * o.z);
    const quat q2 = b.q;
    quat nq = Q(o.w * q2.x + q2.w * o.x + o.y * q2.z - o.z * q2.y,
                o.w * q2.y + q2.w * o.y + o.z * q2.x - o.x * q2.z,
                o.w * q2.z + q2.w * o.z + o.x * q2.y - o.y * q2.x,
                o.w * q2.w - o.x * q2.x - o.y * q2.y - o.z * q2.z);
    return X(np, nq);
}

/* areParallelVectors / areOrthogonalVectors (mathematics_functions.h:76-84) */
static int are_parallel(v3 a, v3 b) { return vlen2(vcross(a, b)) < 0.00001f; }
static int are_orthogonal(v3 a, v3 b) { return fabsf(vdot(a, b)) < 0.001f; }

/* computeClosestPointOnSegment (mathematics_functions.h:96-118) */
static v3 closest_point_on_segment(v3 a, v3 b, v3 c) {
    const v3 ab = vsub(b, a);
    float abl2 = vlen2(ab);
    if (abl2 < MACHINE_EPSILON) return a;
    float t = vdot(vsub(c, a), ab) / abl2;
    if (t < 0.0f) t = 0.0f;
    if (t > 1.0f) t = 1.0f;
    return vadd(a, vmul(ab, t));
}

/* computeClosestPointBetweenTwoSegments (mathematics_functions.h:123-190) */
static void closest_points_segments(v3 s1a, v3 s1b, v3 s2a, v3 s2b, v3* c1, v3* c2) {
    const v3 d1 = vsub(s1b, s1a);
    const v3 d2 = vsub(s2b, s2a);
    const v3 r = vsub(s1a, s2a);
    float a = vlen2(d1);
    float e = vlen2(d2);
    float f = vdot(d2, r);
    float s, t;
    if (a <= MACHINE_EPSILON && e <= MACHINE_EPSILON) { *c1 = s1a; *c2 = s2a; return; }
    if (a <= MACHINE_EPSILON) {
        s = 0.0f;
        t = clampf_std(f / e, 0.0f, 1.0f);
    } else {
        float c = vdot(d1, r);
        if (e <= MACHINE_EPSILON) {
            t = 0.0f;
            s = clampf_std(-c / a, 0.0f, 1.0f);
        } else {
            float b = vdot(d1, d2);
            float denom = a * e - b * b;
            if (denom != 0.0f) s = clampf_std((b * f - c * e) / denom, 0.0f, 1.0f);
            else s = 0.0f;
            t = (b * s + f) / e;
            if (t < 0.0f) { t = 0.0f; s = clampf_std(-c / a, 0.0f, 1.0f); }
            else if (t > 1.0f) { t = 1.0f; s = clampf_std((b - c) / a, 0.0f, 1.0f); }
        }
    }
    *c1 = vadd(s1a, vmul(d1, s));
    *c2 = vadd(s2a, vmul(d2, t));
}

/* computePlaneSegmentIntersection (mathematics_functions.h:224-237) */
static float plane_segment_intersection(v3 a, v3 b, float d, v3 n) {
    const float eps = 0.0001f;
    float t = -1.0f;
    const float nab = vdot(n, vsub(b, a));
    if (fabsf(nab) > eps) t = (d - vdot(n, a)) / nab;
    return t;
}

/* computePointToLineDistance (mathematics_functions.h:240-249) */
static float point_to_line_distance(v3 a, v3 b, v3 p) {
    float dab = vlen(vsub(b, a));
    if (dab < MACHINE_EPSILON) return vlen(vsub(p, a));
    return vlen(vcross(vsub(p, a), vsub(p, b))) / dab;
}

/* projectPointOntoPlane (mathematics_functions.h:396-398) */
static v3 project_onto_plane(v3 p, v3 n, v3 pp) { return vsub(p, vmul(n, vdot(n, vsub(p, pp)))); }

/* ------------------------------------------------------------------ */
/* shapes                                                             */
/* ------------------------------------------------------------------ */
typedef struct { uint32_t vertex, twin, face, next; } hedge;

typedef struct {
    uint32_t nv, nf, nhe;
    float* verts;          /* nv*3 (unscaled) */
    uint32_t* face_start;  /* nf */
    uint32_t* face_count;  /* nf */
    uint32_t* face_verts;  /* sum(face_count) */
    uint32_t* face_edge;   /* nf */
    float* normals;        /* nf*3 unit (ConvexMesh::mFacesNormals) */
    hedge* edges;          /* nhe */
    v3 centroid;
} mesh_t;

typedef struct {
    int32_t mesh;
    v3 scale;
    float* scaled_normals; /* nf*3 (ConvexMeshShape::mScaledFacesNormals) */
} mesh_inst_t;

static mesh_t* g_meshes = NULL;
static uint32_t g_nmeshes = 0;
static mesh_inst_t* g_insts = NULL;
static uint32_t g_ninsts = 0;
static mesh_t g_box; /* box topology (PhysicsCommon::initBoxShapeHalfEdgeStructure) */
static int g_box_ready = 0;

/* HalfEdgeStructure::computeHalfEdges (HalfEdgeStructure.cpp:34-127).  The
 * reference uses hash maps keyed by directed vertex pairs; only their lookup
 * results matter, restated here with dense nv*nv tables. */
static int compute_half_edges(mesh_t* m) {
    const uint32_t nv = m->nv;
    const size_t nn = (size_t)nv * nv;
    int32_t* edge_of_pair = (int32_t*)malloc(nn * sizeof(int32_t));     /* mapEdgeToIndex */
    int32_t* next_pair = (int32_t*)malloc(nn * sizeof(int32_t));        /* nextEdges: pair -> pair */
    uint8_t* seen = (uint8_t*)calloc(nn, 1);                            /* edges map membership */
    hedge* seen_edge = (hedge*)malloc(nn * sizeof(hedge));              /* edges map values */
    uint32_t total = 0;
    for (uint32_t f = 0; f < m->nf; f++) total += m->face_count[f];
    hedge* out = (hedge*)malloc((total + 2) * sizeof(hedge));
    int32_t* key_of_edge = (int32_t*)malloc((total + 2) * sizeof(int32_t)); /* mapEdgeIndexToKey */
    int32_t* face_key = (int32_t*)malloc(m->nf * sizeof(int32_t));          /* mapFaceIndexToEdgeKey */
    uint32_t ne = 0;
    for (size_t i = 0; i < nn; i++) { edge_of_pair[i] = -1; next_pair[i] = -1; }
    for (uint32_t f = 0; f < m->nf; f++) {
        const uint32_t* fv = m->face_verts + m->face_start[f];
        const uint32_t n = m->face_count[f];
        int32_t first_key = 0, prev_key = -1;
        for (uint32_t v = 0; v < n; v++) {
            const uint32_t v1 = fv[v], v2 = fv[v == n - 1 ? 0 : v + 1];
            const int32_t k12 = (int32_t)(v1 * nv + v2), k21 = (int32_t)(v2 * nv + v1);
            hedge e;
            e.face = f; e.vertex = v1; e.twin = 0; e.next = 0;
            if (v == 0) first_key = k12;
            else next_pair[prev_key] = k12;
            if (v == n - 1) next_pair[k12] = first_key;
            seen[k12] = 1; seen_edge[k12] = e;
            face_key[f] = k12;
            if (seen[k21] && edge_of_pair[k21] < 0) {
                const uint32_t idx = ne;
                seen_edge[k21].twin = idx + 1;
                e.twin = idx;
                key_of_edge[idx] = k21;
                key_of_edge[idx + 1] = k12;
                edge_of_pair[k12] = (int32_t)(idx + 1);
                edge_of_pair[k21] = (int32_t)idx;
                out[ne++] = seen_edge[k21];
                out[ne++] = e;
            }
            prev_key = k12;
        }
    }
    int ok = 1;
    for (uint32_t i = 0; i < ne; i++) {
        const int32_t nk = next_pair[key_of_edge[i]];
        if (nk < 0 || edge_of_pair[nk] < 0) { ok = 0; break; }
        out[i].next = (uint32_t)edge_of_pair[nk];
    }
    for (uint32_t f = 0; ok && f < m->nf; f++) {
        if (edge_of_pair[face_key[f]] < 0) { ok = 0; break; }
        m->face_edge[f] = (uint32_t)edge_of_pair[face_key[f]];
    }
    m->edges = out;
    m->nhe = ne;
    free(edge_of_pair); free(next_pair); free(seen); free(seen_edge); free(key_of_edge); free(face_key);
    return ok;
}

static void init_box(void) {
    static const uint32_t faces[24] = {0, 1, 2, 3, 1, 5, 6, 2, 4, 7, 6, 5, 4, 0, 3, 7, 4, 5, 1, 0, 2, 6, 7, 3};
    if (g_box_ready) return;
    memset(&g_box, 0, sizeof(g_box));
    g_box.nv = 8; g_box.nf = 6;
    g_box.face_start = (uint32_t*)malloc(6 * sizeof(uint32_t));
    g_box.face_count = (uint32_t*)malloc(6 * sizeof(uint32_t));
    g_box.face_verts = (uint32_t*)malloc(24 * sizeof(uint32_t));
    g_box.face_edge = (uint32_t*)malloc(6 * sizeof(uint32_t));
    for (int f = 0; f < 6; f++) { g_box.face_start[f] = 4 * f; g_box.face_count[f] = 4; }
    memcpy(g_box.face_verts, faces, sizeof(faces));
    compute_half_edges(&g_box);
    g_box_ready = 1;
}

/* Polyhedron view: a box (half-extents) or a convex mesh instance. */
typedef struct {
    int is_box;
    v3 he;                   /* box */
    const mesh_t* m;         /* topology (box or mesh) */
    const mesh_inst_t* inst; /* mesh only */
} poly_t;

static uint32_t p_nfaces(const poly_t* p) { return p->m->nf; }
static uint32_t p_nhe(const poly_t* p) { return p->m->nhe; }
static hedge p_edge(const poly_t* p, uint32_t e) { return p->m->edges[e]; }
static uint32_t p_face_edge(const poly_t* p, uint32_t f) { return p->m->face_edge[f]; }
static uint32_t p_face_count(const poly_t* p, uint32_t f) { return p->m->face_count[f]; }
static uint32_t p_face_vertex(const poly_t* p, uint32_t f, uint32_t i) { return p->m->face_verts[p->m->face_start[f] + i]; }
/* BoxShape::getVertexPosition (BoxShape.h:192-208); ConvexMeshShape::getVertexPosition (ConvexMeshShape.h:214-217) */
static v3 p_vertex(const poly_t* p, uint32_t v) {
    if (p->is_box) {
        const v3 h = p->he;
        switch (v) {
            case 0: return V(-h.x, -h.y, h.z);
            case 1: return V(h.x, -h.y, h.z);
            case 2: return V(h.x, h.y, h.z);
            case 3: return V(-h.x, h.y, h.z);
            case 4: return V(-h.x, -h.y, -h.z);
            case 5: return V(h.x, -h.y, -h.z);
            case 6: return V(h.x, h.y, -h.z);
            default: return V(-h.x, h.y, -h.z);
        }
    }
    const float* q = p->m->verts + 3 * v;
    return vcmul(V(q[0], q[1], q[2]), p->inst->scale);
}
/* BoxShape::getFaceNormal (BoxShape.h:211-225); ConvexMeshShape::getFaceNormal (ConvexMeshShape.h:220-223) */
static v3 p_normal(const poly_t* p, uint32_t f) {
    if (p->is_box) {
        switch (f) {
            case 0: return V(0, 0, 1);
            case 1: return V(1, 0, 0);
            case 2: return V(0, 0, -1);
            case 3: return V(-1, 0, 0);
            case 4: return V(0, -1, 0);
            default: return V(0, 1, 0);
        }
    }
    const float* n = p->inst->scaled_normals + 3 * f;
    return V(n[0], n[1], n[2]);
}
/* BoxShape::getCentroid (BoxShape.h:228-230); ConvexMeshShape::getCentroid (ConvexMeshShape.h:226-228) */
static v3 p_centroid(const poly_t* p) {
    if (p->is_box) return V(0, 0, 0);
    return vcmul(p->m->centroid, p->inst->scale);
}
/* BoxShape::getLocalSupportPointWithoutMargin (BoxShape.h:166-171);
 * ConvexMeshShape::getLocalSupportPointWithoutMargin (ConvexMeshShape.cpp:80-102) */
static v3 p_support(const poly_t* p, v3 d) {
    if (p->is_box) {
        return V(d.x < 0.0f ? -p->he.x : p->he.x, d.y < 0.0f ? -p->he.y : p->he.y, d.z < 0.0f ? -p->he.z : p->he.z);
    }
    float maxd = DECIMAL_SMALLEST;
    uint32_t imax = 0;
    for (uint32_t i = 0; i < p->m->nv; i++) {
        const float* q = p->m->verts + 3 * i;
        float dp = vdot(d, V(q[0], q[1], q[2]));
        if (dp > maxd) { imax = i; maxd = dp; }
    }
    const float* q = p->m->verts + 3 * imax;
    return vcmul(V(q[0], q[1], q[2]), p->inst->scale);
}
/* ConvexPolyhedronShape::findMostAntiParallelFace (ConvexPolyhedronShape.h:105-123) */
static uint32_t p_most_antiparallel(const poly_t* p, v3 dir) {
    float mind = DECIMAL_LARGEST;
    uint32_t best = 0;
    for (uint32_t i = 0; i < p_nfaces(p); i++) {
        const float d = vdot(p_normal(p, i), dir);
        if (d < mind) { mind = d; best = i; }
    }
    return best;
}

/* Generic convex shape for GJK (sphere, capsule, polyhedron). */
typedef struct {
    int kind;       /* RP3DG_SHAPE_* */
    float radius;   /* sphere/capsule margin */
    float hh;       /* capsule half height */
    poly_t poly;    /* box / mesh */
} cshape_t;

static float c_margin(const cshape_t* s) {
    return (s->kind == RP3DG_SHAPE_SPHERE || s->kind == RP3DG_SHAPE_CAPSULE) ? s->radius : 0.0f;
}
/* getLocalSupportPointWithoutMargin: SphereShape.h:149-153, CapsuleShape.h:191-206 */
static v3 c_support(const cshape_t* s, v3 d) {
    if (s->kind == RP3DG_SHAPE_SPHERE) return V(0, 0, 0);
    if (s->kind == RP3DG_SHAPE_CAPSULE) {
        float top = s->hh * d.y;
        float bottom = -s->hh * d.y;
        if (top > bottom) return V(0, s->hh, 0);
        return V(0, -s->hh, 0);
    }
    return p_support(&s->poly, d);
}
/* ConvexShape::getLocalSupportPointWithMargin (ConvexShape.cpp:40-56) */
static v3 c_support_margin(const cshape_t* s, v3 d) {
    v3 sp = c_support(s, d);
    const float m = c_margin(s);
    if (m != 0.0f) {
        v3 u = V(0.0f, -1.0f, 0.0f);
        if (vlen2(d) > MACHINE_EPSILON * MACHINE_EPSILON) u = vunit(d);
        sp = vadd(sp, vmul(u, m));
    }
    return sp;
}

static int make_shape(const rp3dg_shape* s, cshape_t* out) {
    memset(out, 0, sizeof(*out));
    out->kind = s->kind;
    switch (s->kind) {
        case RP3DG_SHAPE_SPHERE: out->radius = s->params[0]; return 0;
        case RP3DG_SHAPE_CAPSULE: out->radius = s->params[0]; out->hh = s->params[1]; return 0;
        case RP3DG_SHAPE_BOX:
            init_box();
            out->poly.is_box = 1; out->poly.he = V(s->params[0], s->params[1], s->params[2]); out->poly.m = &g_box;
            return 0;
        case RP3DG_SHAPE_CONVEX_MESH:
            if (s->mesh < 0 || (uint32_t)s->mesh >= g_ninsts) return -1;
            out->poly.is_box = 0; out->poly.inst = &g_insts[s->mesh]; out->poly.m = &g_meshes[g_insts[s->mesh].mesh];
            return 0;
    }
    return -1;
}

/* ------------------------------------------------------------------ */
/* narrow-phase item (NarrowPhaseInfoBatch::NarrowPhaseInfo)           */
/* ------------------------------------------------------------------ */
typedef struct { v3 normal, lp1, lp2; float depth; } contact_t;
typedef struct {
    v3 gjk_axis;
    int is_valid, is_obsolete, was_colliding, was_gjk, was_sat, sat_face1, sat_face2;
    uint32_t sat_face, sat_e1, sat_e2;
} lastframe_t;
typedef struct {
    xform t1, t2;
    cshape_t s1, s2;
    int report;
    int is_colliding;
    uint32_t nb;
    contact_t c[MAX_CONTACTS];
    lastframe_t* lf;
} item_t;

/* NarrowPhaseInfoBatch::addContactPoint (NarrowPhaseInfoBatch.h:170-185) */
static void add_contact(item_t* it, v3 n, float depth, v3 lp1, v3 lp2) {
    if (it->nb < MAX_CONTACTS) {
        it->c[it->nb].normal = n; it->c[it->nb].depth = depth; it->c[it->nb].lp1 = lp1; it->c[it->nb].lp2 = lp2;
        it->nb++;
    }
}

/* ------------------------------------------------------------------ */
/* SphereVsSphereAlgorithm::testCollision (SphereVsSphereAlgorithm.cpp:34-113) */
/* ------------------------------------------------------------------ */
static void sphere_sphere(item_t* it) {
    const xform t1 = it->t1, t2 = it->t2;
    v3 d = vsub(t2.p, t1.p);
    float d2 = vlen2(d);
    const float r1 = it->s1.radius, r2 = it->s2.radius;
    const float sum = r1 + r2;
    const float sum2 = sum * sum;
    if (d2 < sum2) {
        const float depth = sum - sqrtf(d2);
        if (depth > 0) {
            if (it->report) {
                const xform i1 = xinv(t1), i2 = xinv(t2);
                v3 p1, p2, n;
                if (d2 > MACHINE_EPSILON) {
                    const v3 c2in1 = xapply(i1, t2.p);
                    const v3 c1in2 = xapply(i2, t1.p);
                    p1 = vmul(vunit(c2in1), r1);
                    p2 = vmul(vunit(c1in2), r2);
                    n = vunit(d);
                } else {
                    n = V(0, 1, 0);
                    p1 = vmul(qrot(i1.q, n), r1);
                    p2 = vmul(qrot(i2.q, n), r2);
                }
                add_contact(it, n, depth, p1, p2);
            }
            it->is_colliding = 1;
        }
    }
}

/* SphereVsCapsuleAlgorithm::testCollision (SphereVsCapsuleAlgorithm.cpp:38-152) */
static void sphere_capsule(item_t* it) {
    const int sphere1 = it->s1.kind == RP3DG_SHAPE_SPHERE;
    const cshape_t* sph = sphere1 ? &it->s1 : &it->s2;
    const cshape_t* cap = sphere1 ? &it->s2 : &it->s1;
    const float capHeight = cap->hh + cap->hh;
    const float sr = sph->radius, cr = cap->radius;
    const xform s2w = sphere1 ? it->t1 : it->t2;
    const xform c2w = sphere1 ? it->t2 : it->t1;
    const xform w2c = xinv(c2w);
    const xform s2c = xmul(w2c, s2w);
    const v3 center = s2c.p;
    const float half = capHeight * 0.5f;
    const v3 segA = V(0, -half, 0), segB = V(0, half, 0);
    const v3 closest = closest_point_on_segment(segA, segB, center);
    v3 c2s = vsub(closest, center);
    const float dist2 = vlen2(c2s);
    float sum = sr + cr;
    if (dist2 < sum * sum) {
        float depth;
        v3 nw, psph, pcap;
        if (it->report) {
            if (dist2 > MACHINE_EPSILON) {
                float dist = sqrtf(dist2);
                c2s = vdivs(c2s, dist);
                psph = xapply(xinv(s2c), vadd(center, vmul(c2s, sr)));
                pcap = vsub(closest, vmul(c2s, cr));
                nw = qrot(c2w.q, c2s);
                depth = sum - dist;
                if (!sphere1) nw = vneg(nw);
            } else {
                v3 seg = vunit(vsub(segB, segA));
                v3 vec1 = V(1, 0, 0), vec2 = V(0, 1, 0);
                float cosA1 = fabsf(seg.x), cosA2 = fabsf(seg.y);
                depth = sum;
                v3 ncap = cosA1 < cosA2 ? vcross(seg, vec1) : vcross(seg, vec2);
                nw = qrot(c2w.q, ncap);
                psph = xapply(xinv(s2c), vadd(center, vmul(ncap, sr)));
                pcap = vsub(center, vmul(ncap, cr));
            }
            if (depth <= 0.0f) return;
            add_contact(it, nw, depth, sphere1 ? psph : pcap, sphere1 ? pcap : psph);
        }
        it->is_colliding = 1;
    }
}

/* CapsuleVsCapsuleAlgorithm::testCollision (CapsuleVsCapsuleAlgorithm.cpp:37-243) */
static void capsule_capsule(item_t* it) {
    const xform c1to2 = xmul(xinv(it->t2), it->t1);
    const float h1 = it->s1.hh + it->s1.hh, h2 = it->s2.hh + it->s2.hh;
    const float r1 = it->s1.radius, r2 = it->s2.radius;
    const float hh1 = h1 * 0.5f;
    v3 s1a = V(0, -hh1, 0), s1b = V(0, hh1, 0);
    s1a = xapply(c1to2, s1a);
    s1b = xapply(c1to2, s1b);
    const float hh2 = h2 * 0.5f;
    const v3 s2a = V(0, -hh2, 0), s2b = V(0, hh2, 0);
    const v3 seg1 = vsub(s1b, s1a), seg2 = vsub(s2b, s2a);
    const float sum = r1 + r2;
    const int parallel = are_parallel(seg1, seg2);
    if (parallel) {
        const float perp = point_to_line_distance(s1a, s1b, s2a);
        if (perp >= sum) return;
        float d1 = vdot(seg1, s1a);
        float d2 = -vdot(seg1, s1b);
        float t1 = plane_segment_intersection(s2b, s2a, d1, seg1);
        float t2 = plane_segment_intersection(s2a, s2b, d2, vneg(seg1));
        if (t1 > 0.0f && t2 > 0.0f) {
            if (it->report) {
                if (t1 > 1.0f) t1 = 1.0f;
                const v3 clipA = vsub(s2b, vmul(seg2, t1));
                if (t2 > 1.0f) t2 = 1.0f;
                const v3 clipB = vadd(s2a, vmul(seg2, t2));
                const v3 seg1n = vunit(seg1);
                v3 onSeg1 = vadd(s1a, vmul(seg1n, vdot(seg1n, vsub(s2a, s1a))));
                v3 n2, s1to2;
                if (perp > MACHINE_EPSILON) {
                    s1to2 = vsub(s2a, onSeg1);
                    n2 = vunit(s1to2);
                } else {
                    v3 vec1 = V(1, 0, 0), vec2 = V(0, 1, 0);
                    v3 seg2n = vunit(seg2);
                    float cosA1 = fabsf(seg2n.x), cosA2 = fabsf(seg2n.y);
                    s1to2 = V(0, 0, 0);
                    n2 = cosA1 < cosA2 ? vcross(seg2n, vec1) : vcross(seg2n, vec2);
                }
                const xform c2to1 = xinv(c1to2);
                const v3 pA1 = xapply(c2to1, vadd(vsub(clipA, s1to2), vmul(n2, r1)));
                const v3 pB1 = xapply(c2to1, vadd(vsub(clipB, s1to2), vmul(n2, r1)));
                const v3 pA2 = vsub(clipA, vmul(n2, r2));
                const v3 pB2 = vsub(clipB, vmul(n2, r2));
                float depth = sum - perp;
                const v3 nw = qrot(it->t2.q, n2);
                add_contact(it, nw, depth, pA1, pA2);
                add_contact(it, nw, depth, pB1, pB2);
            }
            it->is_colliding = 1;
            return;
        }
    }
    v3 cp1, cp2;
    closest_points_segments(s1a, s1b, s2a, s2b, &cp1, &cp2);
    v3 d = vsub(cp2, cp1);
    const float dist2 = vlen2(d);
    if (dist2 < sum * sum) {
        if (it->report) {
            if (dist2 > MACHINE_EPSILON) {
                float dist = sqrtf(dist2);
                d = vdivs(d, dist);
                const v3 p1 = xapply(xinv(c1to2), vadd(cp1, vmul(d, r1)));
                const v3 p2 = vsub(cp2, vmul(d, r2));
                const v3 nw = qrot(it->t2.q, d);
                float depth = fmax_std(sum - dist, MACHINE_EPSILON);
                add_contact(it, nw, depth, p1, p2);
            } else if (parallel) {
                float sq = vlen2(vsub(s1a, cp2));
                v3 extreme = sq > MACHINE_EPSILON ? s1a : s1b;
                v3 n2 = vnormalize(vsub(cp2, extreme));
                const v3 p1 = xapply(xinv(c1to2), vadd(cp1, vmul(n2, r1)));
                const v3 p2 = vsub(cp2, vmul(n2, r2));
                const v3 nw = qrot(it->t2.q, n2);
                add_contact(it, nw, sum, p1, p2);
            } else {
                v3 n2 = vnormalize(vcross(seg1, seg2));
                const v3 p1 = xapply(xinv(c1to2), vadd(cp1, vmul(n2, r1)));
                const v3 p2 = vsub(cp2, vmul(n2, r2));
                const v3 nw = qrot(it->t2.q, n2);
                add_contact(it, nw, sum, p1, p2);
            }
        }
        it->is_colliding = 1;
    }
}

/* ------------------------------------------------------------------ */
/* VoronoiSimplex (VoronoiSimplex.cpp:25-631, VoronoiSimplex.h)        */
/* ------------------------------------------------------------------ */
typedef struct {
    v3 pts[4], sa[4], sb[4];
    int n;
    float bary[4];
    int recompute;
    v3 cp, cpa, cpb;
    int valid;
} simplex_t;

static void sx_init(simplex_t* s) { memset(s, 0, sizeof(*s)); }
static void sx_add(simplex_t* s, v3 p, v3 a, v3 b) {
    s->pts[s->n] = p; s->sa[s->n] = a; s->sb[s->n] = b; s->n++; s->recompute = 1;
}
static void sx_remove(simplex_t* s, int i) {
    s->n--;
    s->pts[i] = s->pts[s->n]; s->sa[i] = s->sa[s->n]; s->sb[i] = s->sb[s->n];
}
static void sx_reduce(simplex_t* s, int bits) {
    if (s->n >= 4 && (bits & 8) == 0) sx_remove(s, 3);
    if (s->n >= 3 && (bits & 4) == 0) sx_remove(s, 2);
    if (s->n >= 2 && (bits & 2) == 0) sx_remove(s, 1);
    if (s->n >= 1 && (bits & 1) == 0) sx_remove(s, 0);
}
static int sx_contains(const simplex_t* s, v3 p) {
    for (int i = 0; i < s->n; i++) if (vlen2(vsub(s->pts[i], p)) <= SIMPLEX_EPS) return 1;
    return 0;
}
static int sx_affinely_dependent(const simplex_t* s) {
    switch (s->n) {
        case 2: return vlen2(vsub(s->pts[1], s->pts[0])) <= SIMPLEX_EPS;
        case 3: return vlen2(vcross(vsub(s->pts[1], s->pts[0]), vsub(s->pts[2], s->pts[0]))) <= SIMPLEX_EPS;
        case 4: return fabsf(vdot(vsub(s->pts[1], s->pts[0]),
                                  vcross(vsub(s->pts[2], s->pts[0]), vsub(s->pts[3], s->pts[0])))) <= SIMPLEX_EPS;
    }
    return 0;
}
static void sx_setbary(simplex_t* s, float a, float b, float c, float d) {
    s->bary[0] = a; s->bary[1] = b; s->bary[2] = c; s->bary[3] = d;
}
static int sx_bary_valid(const simplex_t* s) {
    return s->bary[0] >= 0.0f && s->bary[1] >= 0.0f && s->bary[2] >= 0.0f && s->bary[3] >= 0.0f;
}
/* computeClosestPointOnSegment (VoronoiSimplex.cpp:304-331) */
static void sx_seg(v3 a, v3 b, int* bits, float* t) {
    v3 AP = vneg(a), AB = vsub(b, a);
    float apab = vdot(AP, AB);
    if (apab > 0.0f) {
        float l2 = vlen2(AB);
        if (apab < l2) { *t = apab / l2; *bits = 3; }
        else { *t = 1.0f; *bits = 2; }
    } else { *t = 0.0f; *bits = 1; }
}
/* computeClosestPointOnTriangle (VoronoiSimplex.cpp:336-451) */
static void sx_tri(v3 a, v3 b, v3 c, int* bits, v3* bc) {
    v3 ab = vsub(b, a), ac = vsub(c, a), ap = vneg(a);
    float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) { *bc = V(1.0f, 0, 0); *bits = 1; return; }
    v3 bp = vneg(b);
    float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { *bc = V(0.0f, 1.0f, 0); *bits = 2; return; }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float v = d1 / (d1 - d3);
        *bc = V(1.0f - v, v, 0); *bits = 3; return;
    }
    v3 cp = vneg(c);
    float d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { *bc = V(0.0f, 0.0f, 1.0f); *bits = 4; return; }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float w = d2 / (d2 - d6);
        *bc = V(1.0f - w, 0, w); *bits = 5; return;
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        *bc = V(0.0f, 1.0f - w, w); *bits = 6; return;
    }
    float denom = 1.0f / (va + vb + vc);
    float v = vb * denom, w = vc * denom;
    *bc = V(1 - v - w, v, w);
    *bits = 7;
}
/* testOriginOutsideOfPlane (VoronoiSimplex.cpp:593-611) */
static int sx_outside(v3 a, v3 b, v3 c, v3 d) {
    const v3 n = vcross(vsub(b, a), vsub(c, a));
    float signp = vdot(vneg(a), n);
    float signd = vdot(vsub(d, a), n);
    if (signd * signd < SIMPLEX_EPS * SIMPLEX_EPS) return -1;
    return signp * signd < 0.0f;
}
static int sx_map(int tri, int first, int second, int third) {
    return (((1 & tri) != 0) << first) | (((2 & tri) != 0) << second) | (((4 & tri) != 0) << third);
}
/* computeClosestPointOnTetrahedron (VoronoiSimplex.cpp:456-575) */
static int sx_tet(v3 a, v3 b, v3 c, v3 d, int* bits, float ab[2], float cd[2], int* degenerate) {
    *degenerate = 0;
    *bits = 15;
    ab[0] = ab[1] = cd[0] = cd[1] = 0.0f;
    int oABC = sx_outside(a, b, c, d), oACD = sx_outside(a, c, d, b);
    int oADB = sx_outside(a, d, b, c), oBDC = sx_outside(b, d, c, a);
    if (oABC < 0 || oACD < 0 || oADB < 0 || oBDC < 0) { *degenerate = 1; return 0; }
    if (oABC == 0 && oACD == 0 && oADB == 0 && oBDC == 0) return 1;
    float best = DECIMAL_LARGEST;
    int tb;
    v3 t;
    if (oABC) {
        sx_tri(a, b, c, &tb, &t);
        v3 cp = vadd(vadd(vmul(a, t.x), vmul(b, t.y)), vmul(c, t.z));
        float sd = vlen2(cp);
        if (sd < best) { best = sd; ab[0] = t.x; ab[1] = t.y; cd[0] = t.z; cd[1] = 0.0f; *bits = tb; }
    }
    if (oACD) {
        sx_tri(a, c, d, &tb, &t);
        v3 cp = vadd(vadd(vmul(a, t.x), vmul(c, t.y)), vmul(d, t.z));
        float sd = vlen2(cp);
        if (sd < best) { best = sd; ab[0] = t.x; ab[1] = 0.0f; cd[0] = t.y; cd[1] = t.z; *bits = sx_map(tb, 0, 2, 3); }
    }
    if (oADB) {
        sx_tri(a, d, b, &tb, &t);
        v3 cp = vadd(vadd(vmul(a, t.x), vmul(d, t.y)), vmul(b, t.z));
        float sd = vlen2(cp);
        if (sd < best) { best = sd; ab[0] = t.x; ab[1] = t.z; cd[0] = 0.0f; cd[1] = t.y; *bits = sx_map(tb, 0, 3, 1); }
    }
    if (oBDC) {
        sx_tri(b, d, c, &tb, &t);
        v3 cp = vadd(vadd(vmul(b, t.x), vmul(d, t.y)), vmul(c, t.z));
        float sd = vlen2(cp);
        /* the reference does not update the best distance here (last face) */
        if (sd < best) { ab[0] = 0.0f; ab[1] = t.x; cd[0] = t.z; cd[1] = t.y; *bits = sx_map(tb, 1, 3, 2); }
    }
    return 1;
}
/* recomputeClosestPoint (VoronoiSimplex.cpp:169-299) */
static int sx_recompute(simplex_t* s) {
    if (s->recompute) {
        s->recompute = 0;
        switch (s->n) {
            case 0: s->valid = 0; break;
            case 1:
                s->cp = s->pts[0]; s->cpa = s->sa[0]; s->cpb = s->sb[0];
                sx_setbary(s, 1, 0, 0, 0);
                s->valid = sx_bary_valid(s);
                break;
            case 2: {
                int bits = 0;
                float t;
                sx_seg(s->pts[0], s->pts[1], &bits, &t);
                s->cpa = vadd(s->sa[0], vmul(vsub(s->sa[1], s->sa[0]), t));
                s->cpb = vadd(s->sb[0], vmul(vsub(s->sb[1], s->sb[0]), t));
                s->cp = vsub(s->cpa, s->cpb);
                sx_setbary(s, 1.0f - t, t, 0, 0);
                s->valid = sx_bary_valid(s);
                sx_reduce(s, bits);
                break;
            }
            case 3: {
                int bits = 0;
                v3 bc;
                sx_tri(s->pts[0], s->pts[1], s->pts[2], &bits, &bc);
                s->cpa = vadd(vadd(vmul(s->sa[0], bc.x), vmul(s->sa[1], bc.y)), vmul(s->sa[2], bc.z));
                s->cpb = vadd(vadd(vmul(s->sb[0], bc.x), vmul(s->sb[1], bc.y)), vmul(s->sb[2], bc.z));
                s->cp = vsub(s->cpa, s->cpb);
                sx_setbary(s, bc.x, bc.y, bc.z, 0.0f);
                s->valid = sx_bary_valid(s);
                sx_reduce(s, bits);
                break;
            }
            case 4: {
                int bits = 0, degenerate;
                float ab[2], cd[2];
                int outside = sx_tet(s->pts[0], s->pts[1], s->pts[2], s->pts[3], &bits, ab, cd, &degenerate);
                if (outside) {
                    s->cpa = vadd(vadd(vadd(vmul(s->sa[0], ab[0]), vmul(s->sa[1], ab[1])), vmul(s->sa[2], cd[0])),
                                  vmul(s->sa[3], cd[1]));
                    s->cpb = vadd(vadd(vadd(vmul(s->sb[0], ab[0]), vmul(s->sb[1], ab[1])), vmul(s->sb[2], cd[0])),
                                  vmul(s->sb[3], cd[1]));
                    s->cp = vsub(s->cpa, s->cpb);
                    sx_setbary(s, ab[0], ab[1], cd[0], cd[1]);
                    sx_reduce(s, bits);
                } else {
                    if (degenerate) {
                        s->valid = 0;
                    } else {
                        sx_setbary(s, 0.0f, 0.0f, 0.0f, 0.0f);
                        s->cpa = V(0, 0, 0); s->cpb = V(0, 0, 0); s->cp = V(0, 0, 0);
                        s->valid = 1;
                    }
                    break;
                }
                s->valid = sx_bary_valid(s);
                break;
            }
        }
    }
    return s->valid;
}
static float sx_max_len2(const simplex_t* s) {
    float m = 0.0f;
    for (int i = 0; i < s->n; i++) { float l = vlen2(s->pts[i]); if (l > m) m = l; }
    return m;
}

/* ------------------------------------------------------------------ */
/* GJKAlgorithm::testCollision (GJKAlgorithm.cpp:50-238)              */
/* ------------------------------------------------------------------ */
enum { GJK_SEPARATED = 0, GJK_COLLIDE_IN_MARGIN = 1, GJK_INTERPENETRATE = 2 };

static int gjk(item_t* it) {
    v3 suppA, suppB, w, pA, pB;
    float vDotw, prevDistSquare;
    int contactFound = 0;
    const cshape_t* s1 = &it->s1;
    const cshape_t* s2 = &it->s2;
    const xform t1 = it->t1, t2 = it->t2;
    const xform t1inv = xinv(t1);
    const xform b2to1 = xmul(t1inv, t2);
    const quat rotToB2 = qmul(qinv(t2.q), t1.q);
    const float margin = c_margin(s1) + c_margin(s2);
    const float marginSquare = margin * margin;
    simplex_t sx;
    sx_init(&sx);
    lastframe_t* lf = it->lf;
    v3 v;
    if (lf->is_valid && lf->was_gjk) v = lf->gjk_axis;
    else v = V(0, 1, 0);
    float distSquare = DECIMAL_LARGEST;
    do {
        suppA = c_support(s1, vneg(v));
        suppB = xapply(b2to1, c_support(s2, qrot(rotToB2, v)));
        w = vsub(suppA, suppB);
        vDotw = vdot(v, w);
        if (vDotw > 0.0f && vDotw * vDotw > distSquare * marginSquare) {
            lf->gjk_axis = v;
            return GJK_SEPARATED;
        }
        if (sx_contains(&sx, w) || distSquare - vDotw <= distSquare * REL_ERROR_SQUARE) { contactFound = 1; break; }
        sx_add(&sx, w, suppA, suppB);
        if (sx_affinely_dependent(&sx)) { contactFound = 1; break; }
        int ok = sx_recompute(&sx);
        v = sx.cp;
        if (!ok) { contactFound = 1; break; }
        prevDistSquare = distSquare;
        distSquare = vlen2(v);
        if (prevDistSquare - distSquare <= MACHINE_EPSILON * prevDistSquare) {
            v = sx.cp; /* backupClosestPointInSimplex */
            distSquare = vlen2(v);
            contactFound = 1;
            break;
        }
    } while (sx.n != 4 && distSquare > MACHINE_EPSILON * sx_max_len2(&sx));

    if (contactFound && distSquare > MACHINE_EPSILON) {
        pA = sx.cpa; pB = sx.cpb;
        float dist = sqrtf(distSquare);
        pA = vsub(pA, vmul(v, c_margin(s1) / dist));
        pB = xapply(xinv(b2to1), vadd(pB, vmul(v, c_margin(s2) / dist)));
        v3 normal = qrot(t1.q, vneg(vunit(v)));
        float depth = margin - dist;
        if (depth <= 0.0f) return GJK_SEPARATED;
        if (vlen2(normal) < MACHINE_EPSILON) return GJK_SEPARATED;
        if (it->report) add_contact(it, normal, depth, pA, pB);
        return GJK_COLLIDE_IN_MARGIN;
    }
    return GJK_INTERPENETRATE;
}

/* ------------------------------------------------------------------ */
/* SAT (SATAlgorithm.cpp)                                             */
/* ------------------------------------------------------------------ */

/* testCollisionSphereVsConvexPolyhedron (SATAlgorithm.cpp:58-144) +
 * computePolyhedronFaceVsSpherePenetrationDepth (:147-162) */
static int sat_sphere_poly(item_t* it) {
    const int sphere1 = it->s1.kind == RP3DG_SHAPE_SPHERE;
    const cshape_t* sph = sphere1 ? &it->s1 : &it->s2;
    const poly_t* poly = sphere1 ? &it->s2.poly : &it->s1.poly;
    const xform s2w = sphere1 ? it->t1 : it->t2;
    const xform p2w = sphere1 ? it->t2 : it->t1;
    const xform w2p = xinv(p2w);
    const xform s2p = xmul(w2p, s2w);
    const v3 center = s2p.p;
    float minDepth = DECIMAL_LARGEST;
    uint32_t minFace = 0;
    for (uint32_t f = 0; f < p_nfaces(poly); f++) {
        const v3 n = p_normal(poly, f);
        v3 c2f = vsub(p_vertex(poly, p_face_vertex(poly, f, 0)), center);
        float depth = vdot(c2f, n) + sph->radius;
        if (depth <= 0.0f) return 0;
        if (depth < minDepth) { minDepth = depth; minFace = f; }
    }
    if (it->report) {
        const v3 mn = p_normal(poly, minFace);
        v3 mnw = qrot(p2w.q, mn);
        v3 psph = qrot(xinv(s2w).q, vmul(vneg(mnw), sph->radius));
        v3 ppoly = vadd(center, vmul(mn, minDepth - sph->radius));
        v3 nw = sphere1 ? vneg(mnw) : mnw;
        add_contact(it, nw, minDepth, sphere1 ? psph : ppoly, sphere1 ? ppoly : psph);
    }
    it->is_colliding = 1;
    return 1;
}

/* clipSegmentWithPlanes (mathematics_functions.h:256-326) */
static int clip_segment_planes(v3 a, v3 b, const v3* pp, const v3* pn, uint32_t np, v3* out) {
    v3 in[2], o[2];
    int nin = 2, no = 0;
    in[0] = a; in[1] = b;
    for (uint32_t p = 0; p < np; p++) {
        if (nin == 0) return 0;
        no = 0;
        const v3 v1 = in[0], v2 = in[1];
        float v1n = vdot(vsub(v1, pp[p]), pn[p]);
        float v2n = vdot(vsub(v2, pp[p]), pn[p]);
        if (v2n >= 0.0f) {
            if (v1n < 0.0f) {
                float t = plane_segment_intersection(v1, v2, vdot(pn[p], pp[p]), pn[p]);
                if (t >= 0.0f && t <= 1.0f) o[no++] = vadd(v1, vmul(vsub(v2, v1), t));
                else o[no++] = v2;
            } else {
                o[no++] = v1;
            }
            o[no++] = v2;
        } else {
            if (v1n >= 0.0f) {
                o[no++] = v1;
                float t = plane_segment_intersection(v1, v2, -vdot(pn[p], pp[p]), vneg(pn[p]));
                if (t >= 0.0f && t <= 1.0f) o[no++] = vadd(v1, vmul(vsub(v2, v1), t));
            }
        }
        for (int i = 0; i < no; i++) in[i] = o[i];
        nin = no;
    }
    for (int i = 0; i < no; i++) out[i] = o[i];
    return no;
}

/* computeCapsulePolyhedronFaceContactPoints (SATAlgorithm.cpp:381-470) */
static int capsule_poly_face_contacts(uint32_t refFace, float capR, const poly_t* poly, float depth,
                                      xform p2c, v3 nw, v3 sepAxisCap, v3 segAp, v3 segBp, item_t* it, int cap1) {
    const v3 fn = p_normal(poly, refFace);
    const uint32_t first = p_face_edge(poly, refFace);
    uint32_t e = first;
    v3 pp[64], pn[64];
    uint32_t np = 0;
    do {
        const hedge ed = p_edge(poly, e);
        const hedge tw = p_edge(poly, ed.twin);
        v3 v1 = p_vertex(poly, ed.vertex);
        v3 v2 = p_vertex(poly, tw.vertex);
        v3 dir = vsub(v2, v1);
        v3 cn = vcross(fn, dir);
        if (np < 64) { pp[np] = p_vertex(poly, ed.vertex); pn[np] = cn; np++; }
        e = ed.next;
    } while (e != first);
    v3 clip[2];
    int nc = clip_segment_planes(segAp, segBp, pp, pn, np, clip);
    const v3 delta = vmul(fn, depth - capR);
    int found = 0;
    for (int i = 0; i < nc; i++) {
        const float cd = vdot(vsub(pp[0], clip[i]), fn);
        if (cd > depth - capR - 0.001f) {
            if (!found) it->nb = 0;
            found = 1;
            v3 pPoly = vadd(clip[i], delta);
            v3 pCap = vsub(xapply(p2c, clip[i]), vmul(sepAxisCap, capR));
            add_contact(it, nw, depth, cap1 ? pCap : pPoly, cap1 ? pPoly : pCap);
        }
    }
    return found;
}

/* testCollisionCapsuleVsConvexPolyhedron (SATAlgorithm.cpp:165-319) with
 * computePolyhedronFaceVsCapsulePenetrationDepth (:357-376),
 * computeEdgeVsCapsuleInnerSegmentPenetrationDepth (:322-354),
 * isMinkowskiFaceCapsuleVsEdge (:476-482) */
static int sat_capsule_poly(item_t* it) {
    const int cap1 = it->s1.kind == RP3DG_SHAPE_CAPSULE;
    const cshape_t* cap = cap1 ? &it->s1 : &it->s2;
    const poly_t* poly = cap1 ? &it->s2.poly : &it->s1.poly;
    const xform c2w = cap1 ? it->t1 : it->t2;
    const xform p2w = cap1 ? it->t2 : it->t1;
    const xform p2c = xmul(xinv(c2w), p2w);
    const float height = cap->hh + cap->hh;
    const v3 segA = V(0, -height * 0.5f, 0), segB = V(0, height * 0.5f, 0);
    const v3 segAxis = vsub(segB, segA);
    float minDepth = DECIMAL_LARGEST;
    uint32_t minFace = 0;
    int isFace = 0;
    v3 sepAxis = V(0, 0, 0), sepE1 = V(0, 0, 0), sepE2 = V(0, 0, 0);
    for (uint32_t f = 0; f < p_nfaces(poly); f++) {
        const v3 fn = p_normal(poly, f);
        v3 fnc = qrot(p2c.q, fn);
        const v3 sp = c_support_margin(cap, vneg(fnc));
        const v3 pf = xapply(p2c, p_vertex(poly, p_face_vertex(poly, f, 0)));
        const float depth = vdot(vsub(pf, sp), fnc);
        if (depth <= 0.0f) return 0;
        if (depth < minDepth) { minDepth = depth; minFace = f; isFace = 1; sepAxis = fnc; }
    }
    for (uint32_t e = 0; e < p_nhe(poly); e += 2) {
        const hedge ed = p_edge(poly, e);
        const v3 ev1 = p_vertex(poly, ed.vertex);
        const v3 ev2 = p_vertex(poly, p_edge(poly, ed.next).vertex);
        const v3 edirc = qrot(p2c.q, vsub(ev2, ev1));
        const hedge tw = p_edge(poly, ed.twin);
        const v3 n1 = qrot(p2c.q, p_normal(poly, ed.face));
        const v3 n2 = qrot(p2c.q, p_normal(poly, tw.face));
        if (vdot(segAxis, n1) * vdot(segAxis, n2) < 0.0f) {
            float depth = DECIMAL_LARGEST;
            v3 axis = vcross(segAxis, edirc);
            if (vlen2(axis) >= 0.00001f) {
                const v3 cen = xapply(p2c, p_centroid(poly));
                const v3 pe = xapply(p2c, ev1);
                if (vdot(axis, vsub(pe, cen)) < 0) axis = vneg(axis);
                axis = vnormalize(axis);
                const v3 sp = c_support_margin(cap, vneg(axis));
                depth = vdot(vsub(pe, sp), axis);
            }
            if (depth <= 0.0f) return 0;
            if (depth < minDepth) { minDepth = depth; isFace = 0; sepAxis = axis; sepE1 = ev1; sepE2 = ev2; }
        }
    }
    const xform c2p = xinv(p2c);
    const v3 segAp = xapply(c2p, segA), segBp = xapply(c2p, segB);
    v3 nw = qrot(c2w.q, sepAxis);
    if (cap1) nw = vneg(nw);
    const float capR = cap->radius;
    if (isFace) {
        if (it->report)
            return capsule_poly_face_contacts(minFace, capR, poly, minDepth, p2c, nw, sepAxis, segAp, segBp, it, cap1);
    } else {
        if (it->report) {
            v3 cpEdge, cpSeg;
            closest_points_segments(segAp, segBp, sepE1, sepE2, &cpSeg, &cpEdge);
            v3 pCap = vsub(xapply(p2c, cpSeg), vmul(sepAxis, capR));
            add_contact(it, nw, minDepth, cap1 ? pCap : cpEdge, cap1 ? cpEdge : pCap);
        }
    }
    return 1;
}

/* testSingleFaceDirectionPolyhedronVsPolyhedron (SATAlgorithm.cpp:1087-1110) */
static float sat_single_face(const poly_t* p1, const poly_t* p2, xform p1to2, uint32_t f) {
    const v3 fn = p_normal(p1, f);
    const v3 fn2 = qrot(p1to2.q, fn);
    const v3 sp = p_support(p2, vneg(fn2));
    const v3 fv = xapply(p1to2, p_vertex(p1, p_face_vertex(p1, f, 0)));
    return vdot(vsub(fv, sp), fn2);
}
/* testFacesDirectionPolyhedronVsPolyhedron (SATAlgorithm.cpp:1113-1142) */
static float sat_faces(const poly_t* p1, const poly_t* p2, xform p1to2, uint32_t* minFace) {
    float minDepth = DECIMAL_LARGEST;
    for (uint32_t f = 0; f < p_nfaces(p1); f++) {
        float d = sat_single_face(p1, p2, p1to2, f);
        if (d <= 0.0f) { *minFace = f; return d; }
        if (d < minDepth) { minDepth = d; *minFace = f; }
    }
    return minDepth;
}
/* testGaussMapArcsIntersect (SATAlgorithm.cpp:1180-1191) */
static int gauss_arcs(v3 a, v3 b, v3 c, v3 d, v3 bxa, v3 dxc) {
    const float cba = vdot(c, bxa), dba = vdot(d, bxa), adc = vdot(a, dxc), bdc = vdot(b, dxc);
    return cba * dba < 0.0f && adc * bdc < 0.0f && cba * bdc > 0.0f;
}
/* testEdgesBuildMinkowskiFace (SATAlgorithm.cpp:1146-1172) */
static int sat_minkowski(const poly_t* p1, hedge e1, const poly_t* p2, hedge e2, xform p1to2) {
    const v3 a = qrot(p1to2.q, p_normal(p1, e1.face));
    const v3 b = qrot(p1to2.q, p_normal(p1, p_edge(p1, e1.twin).face));
    const v3 c = p_normal(p2, e2.face);
    const v3 d = p_normal(p2, p_edge(p2, e2.twin).face);
    const v3 e1v1 = p_vertex(p1, e1.vertex);
    const v3 e1v2 = p_vertex(p1, p_edge(p1, e1.twin).vertex);
    const v3 bxa = qrot(p1to2.q, vsub(e1v1, e1v2));
    const v3 e2v1 = p_vertex(p2, e2.vertex);
    const v3 e2v2 = p_vertex(p2, p_edge(p2, e2.twin).vertex);
    const v3 dxc = vsub(e2v1, e2v2);
    return gauss_arcs(a, b, vneg(c), vneg(d), bxa, dxc);
}
/* computeDistanceBetweenEdges (SATAlgorithm.cpp:1040-1083) */
static float sat_edge_distance(v3 e1A, v3 e2A, v3 c1, v3 c2, v3 d1, v3 d2, int shape1Triangle, v3* outAxis) {
    if (are_parallel(d1, d2)) return DECIMAL_LARGEST;
    v3 axis = vunit(vcross(d1, d2));
    float dp;
    if (shape1Triangle) dp = vdot(axis, vsub(e2A, c2));
    else dp = vdot(axis, vsub(c1, e1A));
    if (dp > 0.0f) axis = vneg(axis);
    *outAxis = axis;
    return -vdot(axis, vsub(e2A, e1A));
}

/* clipPolygonWithPlane (mathematics_functions.h:332-393) */
static uint32_t clip_polygon(const v3* in, uint32_t nin, v3 pp, v3 pn, v3* out) {
    uint32_t no = 0;
    uint32_t vs = nin - 1;
    const float pnpp = vdot(pn, pp);
    float vsn = vdot(vsub(in[vs], pp), pn);
    for (uint32_t ve = 0; ve < nin; ve++) {
        const v3 a = in[vs], b = in[ve];
        const float ven = vdot(vsub(b, pp), pn);
        if (ven >= 0.0f) {
            if (vsn < 0.0f) {
                const float t = plane_segment_intersection(a, b, pnpp, pn);
                if (t >= 0.0f && t <= 1.0f) out[no++] = vadd(a, vmul(vsub(b, a), t));
                else out[no++] = b;
            }
            out[no++] = b;
        } else {
            if (vsn >= 0.0f) {
                const float t = plane_segment_intersection(a, b, -pnpp, vneg(pn));
                if (t >= 0.0f && t <= 1.0f) out[no++] = vadd(a, vmul(vsub(b, a), t));
                else out[no++] = a;
            }
        }
        vs = ve;
        vsn = ven;
    }
    return no;
}

#define CLIP_CAP 512
/* computePolyhedronVsPolyhedronFaceContactPoints (SATAlgorithm.cpp:893-1036) */
static int sat_face_contacts(int ref1, const poly_t* p1, const poly_t* p2, xform p1to2, xform p2to1, uint32_t minFace,
                             item_t* it) {
    const poly_t* refP = ref1 ? p1 : p2;
    const poly_t* incP = ref1 ? p2 : p1;
    const xform r2i = ref1 ? p1to2 : p2to1;
    const xform i2r = ref1 ? p2to1 : p1to2;
    const v3 axisR = p_normal(refP, minFace);
    const v3 axisI = qrot(r2i.q, axisR);
    const v3 nw = ref1 ? qrot(it->t1.q, axisR) : vneg(qrot(it->t2.q, axisR));
    const uint32_t incFace = p_most_antiparallel(incP, axisI);
    const uint32_t nInc = p_face_count(incP, incFace);
    static v3 buf1[CLIP_CAP], buf2[CLIP_CAP];
    uint32_t n1 = 0, n2 = 0;
    for (uint32_t i = 0; i < nInc; i++) buf1[n1++] = xapply(i2r, p_vertex(incP, p_face_vertex(incP, incFace, i)));
    const uint32_t firstEdge = p_face_edge(refP, minFace);
    int v1in = 0;
    uint32_t nOut = 0, curIdx;
    hedge cur = p_edge(refP, firstEdge);
    v3 ev1 = p_vertex(refP, cur.vertex);
    do {
        v1in = !v1in;
        const hedge nxt = p_edge(refP, cur.next);
        const v3 ev2 = p_vertex(refP, nxt.vertex);
        const v3 dir = vsub(ev2, ev1);
        const v3 pn = vcross(axisR, dir);
        if (v1in) { n2 = clip_polygon(buf1, n1, ev1, pn, buf2); }
        else { n1 = clip_polygon(buf2, n2, ev1, pn, buf1); }
        curIdx = cur.next;
        cur = nxt;
        ev1 = ev2;
        if (v1in) { n1 = 0; nOut = n2; }
        else { n2 = 0; nOut = n1; }
    } while (curIdx != firstEdge && nOut > 0);
    const v3* clipped = v1in ? buf2 : buf1;
    const uint32_t nClip = v1in ? n2 : n1;
    const v3 refV = p_vertex(refP, p_edge(refP, firstEdge).vertex);
    int found = 0;
    for (uint32_t i = 0; i < nClip; i++) {
        float depth = vdot(vsub(refV, clipped[i]), axisR);
        if (depth > 0.0f) {
            found = 1;
            if (it->report) {
                v3 pInc = xapply(r2i, clipped[i]);
                v3 pRef = project_onto_plane(clipped[i], axisR, refV);
                add_contact(it, nw, depth, ref1 ? pRef : pInc, ref1 ? pInc : pRef);
            }
        }
    }
    return found;
}

/* testCollisionConvexPolyhedronVsConvexPolyhedron (SATAlgorithm.cpp:485-889) */
static int sat_poly_poly(item_t* it, int clipPrev) {
    const poly_t* p1 = &it->s1.poly;
    const poly_t* p2 = &it->s2.poly;
    const xform p1to2 = xmul(xinv(it->t2), it->t1);
    const xform p2to1 = xinv(p1to2);
    float minDepth = DECIMAL_LARGEST;
    uint32_t minFace = 0;
    int isFace = 0, isFace1 = 0;
    uint32_t minE1 = 0, minE2 = 0;
    v3 sE1A = V(0, 0, 0), sE1B = V(0, 0, 0), sE2A = V(0, 0, 0), sE2B = V(0, 0, 0), minEdgeAxis = V(0, 0, 0);
    const int tri1 = 0; /* triangles are not part of this restatement */
    lastframe_t* lf = it->lf;

    if (lf->is_valid && lf->was_sat) {
        if (lf->sat_face1) {
            const float d = sat_single_face(p1, p2, p1to2, lf->sat_face);
            if (!lf->was_colliding && d <= 0.0f) return 0;
            if (lf->was_colliding && clipPrev && d > 0.0f) {
                minDepth = d; minFace = lf->sat_face; isFace = 1; isFace1 = 1;
                if (sat_face_contacts(isFace1, p1, p2, p1to2, p2to1, minFace, it)) {
                    lf->sat_face1 = isFace1; lf->sat_face2 = !isFace1; lf->sat_face = minFace;
                    it->is_colliding = 1;
                    return 1;
                }
            }
        } else if (lf->sat_face2) {
            const float d = sat_single_face(p2, p1, p2to1, lf->sat_face);
            if (!lf->was_colliding && d <= 0.0f) return 0;
            if (lf->was_colliding && clipPrev && d > 0.0f) {
                minDepth = d; minFace = lf->sat_face; isFace = 1; isFace1 = 0;
                if (sat_face_contacts(isFace1, p1, p2, p1to2, p2to1, minFace, it)) {
                    lf->sat_face1 = isFace1; lf->sat_face2 = !isFace1; lf->sat_face = minFace;
                    it->is_colliding = 1;
                    return 1;
                }
            }
        } else {
            const hedge e1 = p_edge(p1, lf->sat_e1);
            const hedge e2 = p_edge(p2, lf->sat_e2);
            const v3 e1A = xapply(p1to2, p_vertex(p1, e1.vertex));
            const v3 e1B = xapply(p1to2, p_vertex(p1, p_edge(p1, e1.next).vertex));
            const v3 d1 = vsub(e1B, e1A);
            const v3 e2A = p_vertex(p2, e2.vertex);
            const v3 e2B = p_vertex(p2, p_edge(p2, e2.next).vertex);
            const v3 d2 = vsub(e2B, e2A);
            if (sat_minkowski(p1, e1, p2, e2, p1to2)) {
                v3 axis;
                const v3 c1 = xapply(p1to2, p_centroid(p1));
                float d = sat_edge_distance(e1A, e2A, c1, p_centroid(p2), d1, d2, tri1, &axis);
                if (!lf->was_colliding && d <= 0.0f) return 0;
                if (lf->was_colliding && clipPrev && d > 0.0f && d < DECIMAL_LARGEST) {
                    v3 cp1, cp2;
                    closest_points_segments(e1A, e1B, e2A, e2B, &cp1, &cp2);
                    const v3 w1 = vsub(cp1, e2A);
                    const v3 w2 = vsub(cp2, e1A);
                    const float l1 = vlen2(d1), l2 = vlen2(d2);
                    float t1 = vdot(w1, d2) / l2;
                    float t2 = vdot(w2, d1) / l1;
                    if (t1 >= 0.0f && t1 <= 1.0f && t2 >= 0.0f && t2 <= 1.0f) {
                        if (it->report) {
                            v3 cp1l = xapply(p2to1, cp1);
                            v3 nw = qrot(it->t2.q, axis);
                            add_contact(it, nw, d, cp1l, cp2);
                        }
                        it->is_colliding = 1;
                        return 1;
                    }
                }
            }
        }
    }

    minDepth = DECIMAL_LARGEST;
    isFace = 0;
    uint32_t f1 = 0, f2 = 0;
    const float d1 = sat_faces(p1, p2, p1to2, &f1);
    if (d1 <= 0.0f) {
        lf->sat_face1 = 1; lf->sat_face2 = 0; lf->sat_face = f1;
        return 0;
    }
    const float d2 = sat_faces(p2, p1, p2to1, &f2);
    if (d2 <= 0.0f) {
        lf->sat_face1 = 0; lf->sat_face2 = 1; lf->sat_face = f2;
        return 0;
    }
    if (d1 < d2 * SAT_REL_TOL + SAT_ABS_TOL) {
        isFace = 1; minDepth = fmin_std(d1, d2); minFace = f1; isFace1 = 1;
    } else {
        isFace = 1; minDepth = fmin_std(d1, d2); minFace = f2; isFace1 = 0;
    }
    int separated = 0;
    for (uint32_t i = 0; i < p_nhe(p1); i += 2) {
        const hedge e1 = p_edge(p1, i);
        const v3 e1A = xapply(p1to2, p_vertex(p1, e1.vertex));
        const v3 e1B = xapply(p1to2, p_vertex(p1, p_edge(p1, e1.next).vertex));
        const v3 dir1 = vsub(e1B, e1A);
        for (uint32_t j = 0; j < p_nhe(p2); j += 2) {
            const hedge e2 = p_edge(p2, j);
            const v3 e2A = p_vertex(p2, e2.vertex);
            const v3 e2B = p_vertex(p2, p_edge(p2, e2.next).vertex);
            const v3 dir2 = vsub(e2B, e2A);
            if (sat_minkowski(p1, e1, p2, e2, p1to2)) {
                v3 axis;
                const v3 c1 = xapply(p1to2, p_centroid(p1));
                float d = sat_edge_distance(e1A, e2A, c1, p_centroid(p2), dir1, dir2, tri1, &axis);
                if (d <= 0.0f) {
                    lf->sat_face1 = 0; lf->sat_face2 = 0; lf->sat_e1 = i; lf->sat_e2 = j;
                    separated = 1;
                    break;
                }
                if ((isFace && d * SAT_REL_TOL + SAT_ABS_TOL < minDepth) || (!isFace && d < minDepth)) {
                    minDepth = d; isFace1 = 0; isFace = 0; minE1 = i; minE2 = j;
                    sE1A = e1A; sE1B = e1B; sE2A = e2A; sE2B = e2B; minEdgeAxis = axis;
                }
            }
        }
        if (separated) break;
    }
    if (separated) return 0;
    if (isFace) {
        int found = sat_face_contacts(isFace1, p1, p2, p1to2, p2to1, minFace, it);
        lf->sat_face1 = isFace1; lf->sat_face2 = !isFace1; lf->sat_face = minFace;
        if (!found) return 0;
    } else {
        if (it->report) {
            v3 cp1, cp2;
            closest_points_segments(sE1A, sE1B, sE2A, sE2B, &cp1, &cp2);
            v3 cp1l = xapply(p2to1, cp1);
            v3 nw = qrot(it->t2.q, minEdgeAxis);
            add_contact(it, nw, minDepth, cp1l, cp2);
        }
        lf->sat_face1 = 0; lf->sat_face2 = 0; lf->sat_e1 = minE1; lf->sat_e2 = minE2;
    }
    it->is_colliding = 1;
    return 1;
}

/* ------------------------------------------------------------------ */
/* algorithm wrappers                                                 */
/* ------------------------------------------------------------------ */

/* SphereVsConvexPolyhedronAlgorithm::testCollision (SphereVsConvexPolyhedronAlgorithm.cpp:38-103) */
static void sphere_poly(item_t* it) {
    int r = gjk(it);
    it->lf->was_gjk = 1; it->lf->was_sat = 0;
    if (r == GJK_COLLIDE_IN_MARGIN) { it->is_colliding = 1; return; }
    if (r == GJK_INTERPENETRATE) {
        sat_sphere_poly(it);
        it->lf->was_gjk = 0; it->lf->was_sat = 1;
    }
}

/* CapsuleVsConvexPolyhedronAlgorithm::testCollision (CapsuleVsConvexPolyhedronAlgorithm.cpp:42-177) */
static void capsule_poly(item_t* it) {
    int r = gjk(it);
    it->lf->was_gjk = 1; it->lf->was_sat = 0;
    if (r == GJK_COLLIDE_IN_MARGIN) {
        if (it->report) {
            const contact_t c0 = it->c[0];
            const int cap1 = it->s1.kind == RP3DG_SHAPE_CAPSULE;
            const cshape_t* cap = cap1 ? &it->s1 : &it->s2;
            const poly_t* poly = cap1 ? &it->s2.poly : &it->s1.poly;
            for (uint32_t f = 0; f < p_nfaces(poly); f++) {
                const xform p2w = cap1 ? it->t2 : it->t1;
                const xform c2w = cap1 ? it->t1 : it->t2;
                const v3 fn = p_normal(poly, f);
                v3 fnw = qrot(p2w.q, fn);
                const v3 segA = V(0, -(cap->hh + cap->hh) * 0.5f, 0), segB = V(0, (cap->hh + cap->hh) * 0.5f, 0);
                v3 segDir = vnormalize(qrot(c2w.q, vsub(segB, segA)));
                /* contactPoint is a reference to contactPoints[0]; it only
                 * changes once contacts are found, after which the loop stops */
                const v3 cn = it->c[0].normal;
                int inDir = vdot(fnw, cn) > 0.0f;
                int inContactDir = (cap1 && !inDir) || (!cap1 && inDir);
                if (inContactDir && are_orthogonal(fnw, segDir) && are_parallel(fnw, cn)) {
                    const xform p2c = xmul(xinv(c2w), p2w);
                    const xform c2p = xinv(p2c);
                    const v3 segAp = xapply(c2p, segA), segBp = xapply(c2p, segB);
                    const v3 sepAxisCap = qrot(p2c.q, fn);
                    if (cap1) fnw = vneg(fnw);
                    int found = capsule_poly_face_contacts(f, cap->radius, poly, it->c[0].depth, p2c, fnw, sepAxisCap,
                                                           segAp, segBp, it, cap1);
                    if (found) break;
                }
            }
            (void)c0;
        }
        it->is_colliding = 1;
        return;
    }
    if (r == GJK_INTERPENETRATE) {
        it->is_colliding = sat_capsule_poly(it);
        it->lf->was_gjk = 0; it->lf->was_sat = 1;
    }
}

/* ------------------------------------------------------------------ */
/* meshes                                                             */
/* ------------------------------------------------------------------ */
int rp3do_create_convex_mesh(const float* vertices, uint32_t nv, const uint32_t* face_indices,
                             const uint32_t* face_sizes, uint32_t nf, int32_t* mesh_id) {
    if (!vertices || !face_indices || !face_sizes || nv == 0 || nf == 0 || nv > 4096) return RP3DG_EINVAL;
    mesh_t m;
    memset(&m, 0, sizeof(m));
    m.nv = nv; m.nf = nf;
    m.verts = (float*)malloc(3 * nv * sizeof(float));
    memcpy(m.verts, vertices, 3 * nv * sizeof(float));
    m.face_start = (uint32_t*)malloc(nf * sizeof(uint32_t));
    m.face_count = (uint32_t*)malloc(nf * sizeof(uint32_t));
    m.face_edge = (uint32_t*)malloc(nf * sizeof(uint32_t));
    uint32_t total = 0;
    for (uint32_t f = 0; f < nf; f++) { m.face_start[f] = total; m.face_count[f] = face_sizes[f]; total += face_sizes[f]; }
    m.face_verts = (uint32_t*)malloc(total * sizeof(uint32_t));
    memcpy(m.face_verts, face_indices, total * sizeof(uint32_t));
    for (uint32_t i = 0; i < total; i++) if (m.face_verts[i] >= nv) return RP3DG_EINVAL;
    if (!compute_half_edges(&m)) return RP3DG_EINVAL;
    /* centroid (ConvexMesh::copyVertices, ConvexMesh.cpp:83-108) */
    v3 c = V(0, 0, 0);
    for (uint32_t i = 0; i < nv; i++) c = vadd(c, V(m.verts[3 * i], m.verts[3 * i + 1], m.verts[3 * i + 2]));
    m.centroid = vdivs(c, (float)nv);
    /* Newell normals (ConvexMesh::computeFacesNormals / computeFaceNormal, ConvexMesh.cpp:185-240) */
    m.normals = (float*)malloc(3 * nf * sizeof(float));
    for (uint32_t f = 0; f < nf; f++) {
        v3 n = V(0, 0, 0);
        const uint32_t cnt = m.face_count[f];
        for (uint32_t i = cnt - 1, j = 0; j < cnt; i = j, j++) {
            const float* a = m.verts + 3 * m.face_verts[m.face_start[f] + i];
            const float* b = m.verts + 3 * m.face_verts[m.face_start[f] + j];
            n = vadd(n, V((a[1] - b[1]) * (a[2] + b[2]), (a[2] - b[2]) * (a[0] + b[0]), (a[0] - b[0]) * (a[1] + b[1])));
        }
        const float l = vlen(n);
        if (l > MACHINE_EPSILON) n = vdivs(n, l);
        m.normals[3 * f] = n.x; m.normals[3 * f + 1] = n.y; m.normals[3 * f + 2] = n.z;
    }
    g_meshes = (mesh_t*)realloc(g_meshes, (g_nmeshes + 1) * sizeof(mesh_t));
    g_meshes[g_nmeshes] = m;
    *mesh_id = (int32_t)g_nmeshes++;
    return 0;
}

int rp3do_create_convex_mesh_shape(int32_t mesh_id, float sx, float sy, float sz, int32_t* instance_id) {
    if (mesh_id < 0 || (uint32_t)mesh_id >= g_nmeshes) return RP3DG_EINVAL;
    const mesh_t* m = &g_meshes[mesh_id];
    mesh_inst_t in;
    in.mesh = mesh_id;
    in.scale = V(sx, sy, sz);
    in.scaled_normals = (float*)malloc(3 * m->nf * sizeof(float));
    /* ConvexMeshShape::computeScaledFacesNormals (ConvexMeshShape.cpp:50-70):
     * 1.0 / scale is evaluated in double and stored as decimal */
    const v3 inv = V((float)(1.0 / (double)sx), (float)(1.0 / (double)sy), (float)(1.0 / (double)sz));
    for (uint32_t f = 0; f < m->nf; f++) {
        v3 n = vcmul(inv, V(m->normals[3 * f], m->normals[3 * f + 1], m->normals[3 * f + 2]));
        const float l = vlen(n);
        n = vdivs(n, l);
        in.scaled_normals[3 * f] = n.x; in.scaled_normals[3 * f + 1] = n.y; in.scaled_normals[3 * f + 2] = n.z;
    }
    g_insts = (mesh_inst_t*)realloc(g_insts, (g_ninsts + 1) * sizeof(mesh_inst_t));
    g_insts[g_ninsts] = in;
    *instance_id = (int32_t)g_ninsts++;
    return 0;
}

int rp3do_get_convex_mesh_tables(int32_t instance_id, uint32_t* nb_vertices, uint32_t* nb_faces,
                                 uint32_t* nb_half_edges, uint32_t* half_edges, float* face_normals,
                                 uint32_t* face_edge, float* centroid, uint32_t cap_he, uint32_t cap_faces) {
    if (instance_id < 0 || (uint32_t)instance_id >= g_ninsts) return RP3DG_EINVAL;
    const mesh_inst_t* in = &g_insts[instance_id];
    const mesh_t* m = &g_meshes[in->mesh];
    *nb_vertices = m->nv; *nb_faces = m->nf; *nb_half_edges = m->nhe;
    if (m->nhe > cap_he || m->nf > cap_faces) return RP3DG_ECAPACITY;
    for (uint32_t e = 0; e < m->nhe; e++) {
        half_edges[4 * e] = m->edges[e].vertex; half_edges[4 * e + 1] = m->edges[e].twin;
        half_edges[4 * e + 2] = m->edges[e].face; half_edges[4 * e + 3] = m->edges[e].next;
    }
    for (uint32_t f = 0; f < m->nf; f++) {
        face_normals[3 * f] = in->scaled_normals[3 * f];
        face_normals[3 * f + 1] = in->scaled_normals[3 * f + 1];
        face_normals[3 * f + 2] = in->scaled_normals[3 * f + 2];
        face_edge[f] = m->face_edge[f];
    }
    const v3 c = vcmul(m->centroid, in->scale);
    centroid[0] = c.x; centroid[1] = c.y; centroid[2] = c.z;
    return 0;
}

void rp3do_reset(void) {
    for (uint32_t i = 0; i < g_nmeshes; i++) {
        free(g_meshes[i].verts); free(g_meshes[i].face_start); free(g_meshes[i].face_count);
        free(g_meshes[i].face_verts); free(g_meshes[i].face_edge); free(g_meshes[i].normals); free(g_meshes[i].edges);
    }
    for (uint32_t i = 0; i < g_ninsts; i++) free(g_insts[i].scaled_normals);
    free(g_meshes); free(g_insts);
    g_meshes = NULL; g_insts = NULL; g_nmeshes = 0; g_ninsts = 0;
}

/* ------------------------------------------------------------------ */
/* batch driver                                                       */
/* ------------------------------------------------------------------ */
static void unpack_lf(const rp3dg_lastframe* c, lastframe_t* l) {
    l->gjk_axis = V(c->gjk_axis[0], c->gjk_axis[1], c->gjk_axis[2]);
    l->is_valid = (c->flags & RP3DG_LF_IS_VALID) != 0;
    l->is_obsolete = (c->flags & RP3DG_LF_IS_OBSOLETE) != 0;
    l->was_colliding = (c->flags & RP3DG_LF_WAS_COLLIDING) != 0;
    l->was_gjk = (c->flags & RP3DG_LF_WAS_USING_GJK) != 0;
    l->was_sat = (c->flags & RP3DG_LF_WAS_USING_SAT) != 0;
    l->sat_face1 = (c->flags & RP3DG_LF_SAT_FACE_POLY1) != 0;
    l->sat_face2 = (c->flags & RP3DG_LF_SAT_FACE_POLY2) != 0;
    l->sat_face = c->sat_face; l->sat_e1 = c->sat_edge1; l->sat_e2 = c->sat_edge2;
}
static void pack_lf(const lastframe_t* l, rp3dg_lastframe* c) {
    c->gjk_axis[0] = l->gjk_axis.x; c->gjk_axis[1] = l->gjk_axis.y; c->gjk_axis[2] = l->gjk_axis.z;
    uint8_t f = 0;
    if (l->is_valid) f |= RP3DG_LF_IS_VALID;
    if (l->is_obsolete) f |= RP3DG_LF_IS_OBSOLETE;
    if (l->was_colliding) f |= RP3DG_LF_WAS_COLLIDING;
    if (l->was_gjk) f |= RP3DG_LF_WAS_USING_GJK;
    if (l->was_sat) f |= RP3DG_LF_WAS_USING_SAT;
    if (l->sat_face1) f |= RP3DG_LF_SAT_FACE_POLY1;
    if (l->sat_face2) f |= RP3DG_LF_SAT_FACE_POLY2;
    c->flags = f;
    c->sat_face = (uint8_t)l->sat_face; c->sat_edge1 = (uint8_t)l->sat_e1; c->sat_edge2 = (uint8_t)l->sat_e2;
}

int rp3do_narrowphase(int algorithm, const rp3dg_shape* shapes, uint32_t nb_shapes, const rp3dg_pair_batch* p,
                      const rp3dg_contact_batch* out, int clip) {
    if (!p || !out || !shapes || algorithm < 1 || algorithm > 6) return RP3DG_EINVAL;
    for (uint32_t i = 0; i < p->n; i++) {
        item_t it;
        lastframe_t lf;
        memset(&it, 0, sizeof(it));
        if (p->cache) unpack_lf(&p->cache[i], &lf);
        else { memset(&lf, 0, sizeof(lf)); lf.gjk_axis = V(0, 1, 0); }
        it.lf = &lf;
        if ((uint32_t)p->shape1[i] >= nb_shapes || (uint32_t)p->shape2[i] >= nb_shapes) return RP3DG_EINVAL;
        if (make_shape(&shapes[p->shape1[i]], &it.s1) || make_shape(&shapes[p->shape2[i]], &it.s2)) return RP3DG_EINVAL;
        it.t1 = X(V(p->pos1[i].x, p->pos1[i].y, p->pos1[i].z), Q(p->rot1[i].x, p->rot1[i].y, p->rot1[i].z, p->rot1[i].w));
        it.t2 = X(V(p->pos2[i].x, p->pos2[i].y, p->pos2[i].z), Q(p->rot2[i].x, p->rot2[i].y, p->rot2[i].z, p->rot2[i].w));
        it.report = p->report_contacts ? p->report_contacts[i] != 0 : 1;
        switch (algorithm) {
            case RP3DG_ALGO_SPHERE_VS_SPHERE: sphere_sphere(&it); break;
            case RP3DG_ALGO_SPHERE_VS_CAPSULE: sphere_capsule(&it); break;
            case RP3DG_ALGO_CAPSULE_VS_CAPSULE: capsule_capsule(&it); break;
            case RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON: sphere_poly(&it); break;
            case RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON: capsule_poly(&it); break;
            case RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON:
                sat_poly_poly(&it, clip);
                lf.was_sat = 1; lf.was_gjk = 0; /* ConvexPolyhedronVsConvexPolyhedronAlgorithm.cpp:53-61 */
                break;
        }
        out->is_colliding[i] = (uint8_t)(it.is_colliding ? 1 : 0);
        const uint32_t nc = it.nb < out->max_contacts ? it.nb : out->max_contacts;
        out->nb_contacts[i] = (uint8_t)nc;
        for (uint32_t c = 0; c < nc; c++) {
            const size_t o = (size_t)c * p->n + i;
            out->normal_depth[o].x = it.c[c].normal.x; out->normal_depth[o].y = it.c[c].normal.y;
            out->normal_depth[o].z = it.c[c].normal.z; out->normal_depth[o].w = it.c[c].depth;
            out->local1[o].x = it.c[c].lp1.x; out->local1[o].y = it.c[c].lp1.y; out->local1[o].z = it.c[c].lp1.z;
            out->local1[o].w = 0.0f;
            out->local2[o].x = it.c[c].lp2.x; out->local2[o].y = it.c[c].lp2.y; out->local2[o].z = it.c[c].lp2.z;
            out->local2[o].w = 0.0f;
        }
        if (p->cache) pack_lf(&lf, &p->cache[i]);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* contact manifold of a convex pair (CollisionDetectionSystem.cpp)    */
/* ------------------------------------------------------------------ */
#define MAX_POINTS_IN_MANIFOLD 4                      /* configuration.h:143 */
static const float SAME_POINT_DIST = 0.01f;           /* configuration.h:146 */

static void remove_at(uint32_t* a, uint32_t idx, uint32_t* size) { a[idx] = a[*size - 1]; (*size)--; }

/* reduceContactPoints (CollisionDetectionSystem.cpp:1483-1662); idx[] holds
 * the manifold's point indices (slots), nb > 4 on entry, 4 on exit */
static void reduce_points(uint32_t* idx, uint32_t* nb, const v3* lp1, v3 normal0_world, quat q1) {
    uint32_t cand[RP3DG_MAX_CONTACTS_PER_PAIR];
    uint32_t ncand = *nb;
    for (uint32_t i = 0; i < ncand; i++) cand[i] = idx[i];
    uint32_t keep[4] = {0, 0, 0, 0};
    const v3 nLocal = qrot(qinv(q1), normal0_world);
    /* first point: max (1,1,1) . localPoint1 */
    float maxDot = DECIMAL_SMALLEST;
    uint32_t k = 0;
    for (uint32_t i = 0; i < ncand; i++) {
        const float d = vdot(V(1, 1, 1), lp1[cand[i]]);
        if (d > maxDot) { maxDot = d; k = i; }
    }
    keep[0] = cand[k];
    remove_at(cand, k, &ncand);
    /* second: farthest from the first (>=) */
    float maxDist = 0.0f;
    k = 0;
    for (uint32_t i = 0; i < ncand; i++) {
        const float d = vlen2(vsub(lp1[keep[0]], lp1[cand[i]]));
        if (d >= maxDist) { maxDist = d; k = i; }
    }
    keep[1] = cand[k];
    remove_at(cand, k, &ncand);
    /* third: largest positive or negative area */
    uint32_t kmax = 0, kmin = 0;
    float minArea = 0.0f, maxArea = 0.0f;
    int prevPositive;
    for (uint32_t i = 0; i < ncand; i++) {
        const v3 a = vsub(lp1[keep[0]], lp1[cand[i]]);
        const v3 b = vsub(lp1[keep[1]], lp1[cand[i]]);
        const float area = vdot(vcross(a, b), nLocal);
        if (area >= maxArea) { maxArea = area; kmax = i; }
        if (area <= minArea) { minArea = area; kmin = i; }
    }
    if (maxArea > (-minArea)) { prevPositive = 1; keep[2] = cand[kmax]; remove_at(cand, kmax, &ncand); }
    else { prevPositive = 0; keep[2] = cand[kmin]; remove_at(cand, kmin, &ncand); }
    /* fourth: largest area of opposite winding over the triangle's edges */
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
    *nb = 4;
}

/* removeDuplicatedContactPointsInManifold (CollisionDetectionSystem.cpp:1673-1705) */
static void remove_duplicates(uint32_t* idx, uint32_t* nb, const v3* lp1) {
    const float thr = SAME_POINT_DIST * SAME_POINT_DIST;
    for (uint32_t i = 0; i < *nb; i++) {
        for (uint32_t j = i + 1; j < *nb; j++) {
            const float d = vlen2(vsub(lp1[idx[j]], lp1[idx[i]]));
            if (d < thr) {
                idx[j] = idx[*nb - 1];
                (*nb)--;
                j--;
            }
        }
    }
}

/* The manifold of each colliding convex pair (processPotentialContacts,
 * CollisionDetectionSystem.cpp:1198-1391, convex branch: one manifold holding
 * every point), reduced to at most 4 points and de-duplicated
 * (reducePotentialContactManifolds, :1394-1458).  Rewrites the contact slots
 * of every pair in place (kept points first, in manifold order) and
 * nb_contacts; kept[4*i..] receives the original slot of each kept point. */
int rp3do_reduce_contacts(const rp3dg_pair_batch* p, const rp3dg_contact_batch* c, uint8_t* kept) {
    if (!p || !c) return RP3DG_EINVAL;
    const uint32_t n = p->n;
    for (uint32_t i = 0; i < n; i++) {
        if (p->cache) {
            /* processPotentialContacts, CollisionDetectionSystem.cpp:1209-1217 */
            uint8_t f = p->cache[i].flags;
            f = (uint8_t)((f | RP3DG_LF_IS_VALID) & ~RP3DG_LF_WAS_COLLIDING);
            if (c->is_colliding[i]) f |= RP3DG_LF_WAS_COLLIDING;
            p->cache[i].flags = f;
        }
        uint32_t nb = c->nb_contacts[i];
        uint32_t idx[RP3DG_MAX_CONTACTS_PER_PAIR];
        v3 lp1[RP3DG_MAX_CONTACTS_PER_PAIR];
        for (uint32_t k = 0; k < nb; k++) {
            idx[k] = k;
            const rp3dg_float4 l = c->local1[(size_t)k * n + i];
            lp1[k] = V(l.x, l.y, l.z);
        }
        if (nb > 0 && c->is_colliding[i]) {
            if (nb > MAX_POINTS_IN_MANIFOLD) {
                const rp3dg_float4 nd = c->normal_depth[i];
                reduce_points(idx, &nb, lp1, V(nd.x, nd.y, nd.z), Q(p->rot1[i].x, p->rot1[i].y, p->rot1[i].z, p->rot1[i].w));
            }
            remove_duplicates(idx, &nb, lp1);
        }
        rp3dg_float4 nd[4], l1[4], l2[4];
        const uint32_t m = nb < 4 ? nb : 4;
        for (uint32_t k = 0; k < m; k++) {
            nd[k] = c->normal_depth[(size_t)idx[k] * n + i];
            l1[k] = c->local1[(size_t)idx[k] * n + i];
            l2[k] = c->local2[(size_t)idx[k] * n + i];
        }
        for (uint32_t k = 0; k < m; k++) {
            c->normal_depth[(size_t)k * n + i] = nd[k];
            c->local1[(size_t)k * n + i] = l1[k];
            c->local2[(size_t)k * n + i] = l2[k];
        }
        if (kept) for (uint32_t k = 0; k < 4; k++) kept[4 * (size_t)i + k] = (uint8_t)(k < m ? idx[k] : 255);
        c->nb_contacts[i] = (uint8_t)m;
    }
    return 0;
}

/* ===================================================================== */
/* Dynamics stage of a world step (PhysicsWorld.cpp:310-360,             */
/* DynamicsSystem.cpp:44-183, ContactSolverSystem.cpp:66-818), restated  */
/* phase by phase over the whole world, with the reference's sequential  */
/* order: all islands' manifolds in one pass per phase.                  */
/* ===================================================================== */

typedef struct {
    int b1, b2, nb;
    float im1, im2, friction;
    v3 lf1, lf2, af1, af2;
    float I1[9], I2[9];
    v3 normal, fp1, fp2, r1f, r2f, ofv1, ofv2, fv1, fv2, r1ct1, r1ct2, r2ct1, r2ct2;
    float inv_f1, inv_f2, inv_tw, f1, f2, ftw;
    uint32_t ext;        /* index of the external manifold */
} DynMan;

typedef struct {
    v3 r1, r2, normal, i1, i2;
    float depth, inv_mass, restitution_bias, impulse, split_impulse;
    int resting;
    uint32_t ext;        /* index of the external contact point */
} DynPt;

static v3 L4(rp3dg_float4 a) { return V(a.x, a.y, a.z); }
static rp3dg_float4 S4(v3 a) { rp3dg_float4 r; r.x = a.x; r.y = a.y; r.z = a.z; r.w = 0.0f; return r; }
/* Matrix3x3 * Vector3 (Matrix3x3.h:324-331) */
static v3 m3v(const float* m, v3 v) {
    return V(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
             m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
/* Quaternion::getMatrix (Quaternion.cpp:138-165) */
static void q_matrix(quat q, float* r) {
    float nQ = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w, s = 0.0f;
    if (nQ > 0.0f) s = 2.0f / nQ;
    float xs = q.x * s, ys = q.y * s, zs = q.z * s, wxs = q.w * xs, wys = q.w * ys, wzs = q.w * zs;
    float xxs = q.x * xs, xys = q.x * ys, xzs = q.x * zs, yys = q.y * ys, yzs = q.y * zs, zzs = q.z * zs;
    r[0] = 1.0f - yys - zzs; r[1] = xys - wzs; r[2] = xzs + wys;
    r[3] = xys + wzs; r[4] = 1.0f - xxs - zzs; r[5] = yzs - wxs;
    r[6] = xzs - wys; r[7] = yzs + wxs; r[8] = 1.0f - xxs - yys;
}
/* Matrix3x3 * Matrix3x3 (Matrix3x3.h:302-321) */
static void m3m(const float* a, const float* b, float* o) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) o[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}
/* deltaV of ContactSolverSystem.cpp:196-201 */
static v3 rel_vel(v3 v1, v3 w1, v3 v2, v3 w2, v3 r1, v3 r2) {
    return V(v2.x + w2.y * r2.z - w2.z * r2.y - v1.x - w1.y * r1.z + w1.z * r1.y,
             v2.y + w2.z * r2.x - w2.x * r2.z - v1.y - w1.z * r1.x + w1.x * r1.z,
             v2.z + w2.x * r2.y - w2.y * r2.x - v1.z - w1.x * r1.y + w1.y * r1.x);
}
/* Vector3::getOneUnitOrthogonalVector (Vector3.cpp:46-64) */
static v3 one_unit_orthogonal(v3 v) {
    v3 a = V(fabsf(v.x), fabsf(v.y), fabsf(v.z));
    int k = (a.x < a.y ? (a.x < a.z ? 0 : 2) : (a.y < a.z ? 1 : 2));
    if (k == 0) return vdivs(V(0.0f, -v.z, v.y), sqrtf(v.y * v.y + v.z * v.z));
    if (k == 1) return vdivs(V(-v.z, 0.0f, v.x), sqrtf(v.x * v.x + v.z * v.z));
    return vdivs(V(-v.y, v.x, 0.0f), sqrtf(v.x * v.x + v.y * v.y));
}
/* v -= s * imp * lock (or +=), Vector3 operators */
static v3 lin_sub(v3 v, float s, v3 imp, v3 lock) { return vsub(v, vcmul(vmul(imp, s), lock)); }
static v3 lin_add(v3 v, float s, v3 imp, v3 lock) { return vadd(v, vcmul(vmul(imp, s), lock)); }

int rp3do_dynamics_step(const rp3dg_dynamics_params* pr, const rp3dg_bodies* B, const rp3dg_colliders* Cl,
                        const rp3dg_manifolds* M, const rp3dg_points* P, const rp3dg_islands* IS) {
    const uint32_t nb = B->n, ne = B->n_enabled;
    const float dt = pr->dt;
    v3* cv = (v3*)calloc(nb ? nb : 1, sizeof(v3));
    v3* cw = (v3*)calloc(nb ? nb : 1, sizeof(v3));
    v3* sv = (v3*)calloc(nb ? nb : 1, sizeof(v3));
    v3* sw = (v3*)calloc(nb ? nb : 1, sizeof(v3));
    DynMan* man = (DynMan*)calloc(M->n ? M->n : 1, sizeof(DynMan));
    DynPt* pt = (DynPt*)calloc(P->n ? P->n : 1, sizeof(DynPt));
    if (!cv || !cw || !sv || !sw || !man || !pt) { free(cv); free(cw); free(sv); free(sw); free(man); free(pt); return RP3DG_ENOMEM; }
    /* bodies outside the enabled range keep their stored velocities */
    for (uint32_t i = ne; i < nb; i++) { cv[i] = L4(B->linear_velocity[i]); cw[i] = L4(B->angular_velocity[i]); }

    /* updateBodiesInverseWorldInertiaTensors (PhysicsWorld.cpp:310-318) */
    for (uint32_t i = 0; i < ne; i++) {
        float R[9], D[9], W[9];
        rp3dg_float4 o = B->orientation[i];
        q_matrix(Q(o.x, o.y, o.z, o.w), R);
        v3 inv = L4(B->inv_inertia_local[i]);
        D[0] = R[0] * inv.x; D[1] = R[3] * inv.x; D[2] = R[6] * inv.x;
        D[3] = R[1] * inv.y; D[4] = R[4] * inv.y; D[5] = R[7] * inv.y;
        D[6] = R[2] * inv.z; D[7] = R[5] * inv.z; D[8] = R[8] * inv.z;
        m3m(R, D, W);
        for (int r = 0; r < 3; r++) {
            rp3dg_float4 row; row.x = W[3 * r]; row.y = W[3 * r + 1]; row.z = W[3 * r + 2]; row.w = 0.0f;
            B->inv_inertia_world[3 * i + r] = row;
        }
    }
    /* integrateRigidBodiesVelocities (DynamicsSystem.cpp:117-183) */
    for (uint32_t i = 0; i < ne; i++) {
        const rp3dg_float4 m = B->mass[i];
        const float* W = &B->inv_inertia_world[3 * i].x;
        float I[9] = {W[0], W[1], W[2], W[4], W[5], W[6], W[8], W[9], W[10]};
        v3 lf = L4(B->linear_lock[i]), af = L4(B->angular_lock[i]);
        cv[i] = vadd(L4(B->linear_velocity[i]), vcmul(vmul(lf, dt * m.y), L4(B->force[i])));
        cw[i] = vadd(L4(B->angular_velocity[i]), vcmul(vmul(af, dt), m3v(I, L4(B->torque[i]))));
    }
    if (pr->gravity_enabled)
        for (uint32_t i = 0; i < ne; i++)
            if (B->gravity[i]) {
                const rp3dg_float4 m = B->mass[i];
                v3 g = V(pr->gravity[0], pr->gravity[1], pr->gravity[2]);
                cv[i] = vadd(cv[i], vcmul(vmul(vmul(L4(B->linear_lock[i]), dt * m.y), m.x), g));
            }
    for (uint32_t i = 0; i < ne; i++) {
        const rp3dg_float4 m = B->mass[i];
        float ld = 1.0f / (1.0f + m.z * dt), ad = 1.0f / (1.0f + m.w * dt);
        cv[i] = vmul(cv[i], ld);
        cw[i] = vmul(cw[i], ad);
    }

    /* ContactSolverSystem::init / initializeForIsland (:66-318) */
    uint32_t nm = 0, np = 0;
    for (uint32_t il = 0; il < IS->n; il++) {
        for (uint32_t e = IS->manifold_start[il]; e < IS->manifold_start[il] + IS->manifold_count[il]; e++) {
            DynMan* c = &man[nm];
            const int32_t* id = &M->ids[4 * e];
            const int b1 = id[0], b2 = id[1], c1 = id[2], c2 = id[3];
            c->b1 = b1; c->b2 = b2; c->nb = M->nb_points[e]; c->ext = e;
            v3 x1 = L4(B->com_world[b1]), x2 = L4(B->com_world[b2]);
            for (int k = 0; k < 9; k++) {
                c->I1[k] = (&B->inv_inertia_world[3 * b1].x)[(k / 3) * 4 + k % 3];
                c->I2[k] = (&B->inv_inertia_world[3 * b2].x)[(k / 3) * 4 + k % 3];
            }
            c->im1 = B->mass[b1].y; c->im2 = B->mass[b2].y;
            c->lf1 = L4(B->linear_lock[b1]); c->lf2 = L4(B->linear_lock[b2]);
            c->af1 = L4(B->angular_lock[b1]); c->af2 = L4(B->angular_lock[b2]);
            c->friction = Cl->material[c1].x * Cl->material[c2].x;
            c->normal = V(0.0f, 0.0f, 0.0f); c->fp1 = V(0.0f, 0.0f, 0.0f); c->fp2 = V(0.0f, 0.0f, 0.0f);
            v3 v1 = L4(B->linear_velocity[b1]), w1 = L4(B->angular_velocity[b1]);
            v3 v2 = L4(B->linear_velocity[b2]), w2 = L4(B->angular_velocity[b2]);
            rp3dg_float4 o1 = Cl->world_orientation[c1], o2 = Cl->world_orientation[c2];
            xform t1 = X(L4(Cl->world_position[c1]), Q(o1.x, o1.y, o1.z, o1.w));
            xform t2 = X(L4(Cl->world_position[c2]), Q(o2.x, o2.y, o2.z, o2.w));
            for (uint32_t q = M->point_start[e]; q < M->point_start[e] + c->nb; q++) {
                DynPt* p = &pt[np];
                p->ext = q;
                p->normal = L4(P->normal_depth[q]);
                v3 p1 = xapply(t1, L4(P->local1[q])), p2 = xapply(t2, L4(P->local2[q]));
                p->r1 = V(p1.x - x1.x, p1.y - x1.y, p1.z - x1.z);
                p->r2 = V(p2.x - x2.x, p2.y - x2.y, p2.z - x2.z);
                p->depth = P->normal_depth[q].w;
                p->resting = P->is_resting[q];
                P->is_resting[q] = 1;
                p->impulse = P->penetration_impulse[q];
                p->split_impulse = 0.0f;
                c->fp1 = V(c->fp1.x + p1.x, c->fp1.y + p1.y, c->fp1.z + p1.z);
                c->fp2 = V(c->fp2.x + p2.x, c->fp2.y + p2.y, c->fp2.z + p2.z);
                v3 dv = rel_vel(v1, w1, v2, w2, p->r1, p->r2);
                v3 r1n = vcross(p->r1, p->normal), r2n = vcross(p->r2, p->normal);
                p->i1 = m3v(c->I1, r1n);
                p->i2 = m3v(c->I2, r2n);
                float mp = c->im1 + c->im2 + vdot(vcross(p->i1, p->r1), p->normal) + vdot(vcross(p->i2, p->r2), p->normal);
                p->inv_mass = mp > 0.0f ? 1.0f / mp : 0.0f;
                p->restitution_bias = 0.0f;
                float dvn = dv.x * p->normal.x + dv.y * p->normal.y + dv.z * p->normal.z;
                float b1r = Cl->material[c1].y, b2r = Cl->material[c2].y;
                float rest = (b1r > b2r) ? b1r : b2r;
                if (dvn < -pr->restitution_velocity_threshold) p->restitution_bias = rest * dvn;
                c->normal = V(c->normal.x + p->normal.x, c->normal.y + p->normal.y, c->normal.z + p->normal.z);
                np++;
            }
            c->fp1 = vdivs(c->fp1, (float)c->nb);
            c->fp2 = vdivs(c->fp2, (float)c->nb);
            c->r1f = V(c->fp1.x - x1.x, c->fp1.y - x1.y, c->fp1.z - x1.z);
            c->r2f = V(c->fp2.x - x2.x, c->fp2.y - x2.y, c->fp2.z - x2.z);
            c->ofv1 = L4(M->friction_vector1[e]);
            c->ofv2 = L4(M->friction_vector2[e]);
            c->f1 = M->friction_impulse[e].x; c->f2 = M->friction_impulse[e].y; c->ftw = M->friction_impulse[e].z;
            c->normal = vnormalize(c->normal);
            v3 dvf = rel_vel(v1, w1, v2, w2, c->r1f, c->r2f);
            /* computeFrictionVectors (:789-818) */
            v3 nv = vmul(c->normal, vdot(dvf, c->normal));
            v3 tv = V(dvf.x - nv.x, dvf.y - nv.y, dvf.z - nv.z);
            float lt = vlen(tv);
            c->fv1 = lt > MACHINE_EPSILON ? vdivs(tv, lt) : one_unit_orthogonal(c->normal);
            c->fv2 = vcross(c->normal, c->fv1);
            c->r1ct1 = vcross(c->r1f, c->fv1); c->r1ct2 = vcross(c->r1f, c->fv2);
            c->r2ct1 = vcross(c->r2f, c->fv1); c->r2ct2 = vcross(c->r2f, c->fv2);
            float f1m = c->im1 + c->im2 + vdot(vcross(m3v(c->I1, c->r1ct1), c->r1f), c->fv1) +
                        vdot(vcross(m3v(c->I2, c->r2ct1), c->r2f), c->fv1);
            float f2m = c->im1 + c->im2 + vdot(vcross(m3v(c->I1, c->r1ct2), c->r1f), c->fv2) +
                        vdot(vcross(m3v(c->I2, c->r2ct2), c->r2f), c->fv2);
            float twm = vdot(c->normal, m3v(c->I1, c->normal)) + vdot(c->normal, m3v(c->I2, c->normal));
            c->inv_f1 = f1m > 0.0f ? 1.0f / f1m : 0.0f;
            c->inv_f2 = f2m > 0.0f ? 1.0f / f2m : 0.0f;
            c->inv_tw = twm > 0.0f ? 1.0f / twm : 0.0f;
            nm++;
        }
    }

    /* warmStart (:324-476) */
    uint32_t pi_ = 0;
    for (uint32_t k = 0; k < nm; k++) {
        DynMan* c = &man[k];
        const int b1 = c->b1, b2 = c->b2;
        int any = 0;
        for (int i = 0; i < c->nb; i++, pi_++) {
            DynPt* p = &pt[pi_];
            if (p->resting) {
                any = 1;
                v3 ip = V(p->normal.x * p->impulse, p->normal.y * p->impulse, p->normal.z * p->impulse);
                cv[b1].x -= c->im1 * ip.x * c->lf1.x; cv[b1].y -= c->im1 * ip.y * c->lf1.y; cv[b1].z -= c->im1 * ip.z * c->lf1.z;
                cw[b1].x -= p->i1.x * c->af1.x * p->impulse; cw[b1].y -= p->i1.y * c->af1.y * p->impulse;
                cw[b1].z -= p->i1.z * c->af1.z * p->impulse;
                cv[b2].x += c->im2 * ip.x * c->lf2.x; cv[b2].y += c->im2 * ip.y * c->lf2.y; cv[b2].z += c->im2 * ip.z * c->lf2.z;
                cw[b2].x += p->i2.x * c->af2.x * p->impulse; cw[b2].y += p->i2.y * c->af2.y * p->impulse;
                cw[b2].z += p->i2.z * c->af2.z * p->impulse;
            } else {
                p->impulse = 0.0f;
            }
        }
        if (any) {
            v3 ofi = V(c->f1 * c->ofv1.x + c->f2 * c->ofv2.x, c->f1 * c->ofv1.y + c->f2 * c->ofv2.y,
                       c->f1 * c->ofv1.z + c->f2 * c->ofv2.z);
            c->f1 = vdot(ofi, c->fv1);
            c->f2 = vdot(ofi, c->fv2);
            v3 a1 = V(-c->r1ct1.x * c->f1, -c->r1ct1.y * c->f1, -c->r1ct1.z * c->f1);
            v3 l2 = V(c->fv1.x * c->f1, c->fv1.y * c->f1, c->fv1.z * c->f1);
            v3 a2 = V(c->r2ct1.x * c->f1, c->r2ct1.y * c->f1, c->r2ct1.z * c->f1);
            cv[b1] = lin_sub(cv[b1], c->im1, l2, c->lf1);
            cw[b1] = vadd(cw[b1], vcmul(c->af1, m3v(c->I1, a1)));
            cv[b2] = lin_add(cv[b2], c->im2, l2, c->lf2);
            cw[b2] = vadd(cw[b2], vcmul(c->af2, m3v(c->I2, a2)));
            a1 = V(-c->r1ct2.x * c->f2, -c->r1ct2.y * c->f2, -c->r1ct2.z * c->f2);
            l2 = V(c->fv2.x * c->f2, c->fv2.y * c->f2, c->fv2.z * c->f2);
            a2 = V(c->r2ct2.x * c->f2, c->r2ct2.y * c->f2, c->r2ct2.z * c->f2);
            cv[b1] = lin_sub(cv[b1], c->im1, l2, c->lf1);
            cw[b1] = vadd(cw[b1], vcmul(c->af1, m3v(c->I1, a1)));
            cv[b2] = lin_add(cv[b2], c->im2, l2, c->lf2);
            cw[b2] = vadd(cw[b2], vcmul(c->af2, m3v(c->I2, a2)));
            a1 = V(-c->normal.x * c->ftw, -c->normal.y * c->ftw, -c->normal.z * c->ftw);
            a2 = V(c->normal.x * c->ftw, c->normal.y * c->ftw, c->normal.z * c->ftw);
            cw[b1] = vadd(cw[b1], vcmul(c->af1, m3v(c->I1, a1)));
            cw[b2] = vadd(cw[b2], vcmul(c->af2, m3v(c->I2, a2)));
            cw[b1] = vsub(cw[b1], vcmul(c->af1, m3v(c->I1, a2)));
            cw[b2] = vadd(cw[b2], vcmul(c->af2, m3v(c->I2, a2)));
        } else {
            c->f1 = 0.0f; c->f2 = 0.0f; c->ftw = 0.0f;
        }
    }

    /* solve (:479-759), velocity iterations (PhysicsWorld.cpp:333-339) */
    const float beta = pr->split_impulse ? 0.2f : 0.2f;   /* BETA_SPLIT_IMPULSE : BETA (:43-44) */
    const float SLOP = 0.01f;                             /* :45 */
    for (int it = 0; it < pr->velocity_iterations; it++) {
        uint32_t q = 0;
        for (uint32_t k = 0; k < nm; k++) {
            DynMan* c = &man[k];
            const int b1 = c->b1, b2 = c->b2;
            float sum = 0.0f;
            for (int i = 0; i < c->nb; i++, q++) {
                DynPt* p = &pt[q];
                v3 dv = rel_vel(cv[b1], cw[b1], cv[b2], cw[b2], p->r1, p->r2);
                float Jv = dv.x * p->normal.x + dv.y * p->normal.y + dv.z * p->normal.z;
                float bias = 0.0f;
                if (p->depth > SLOP) bias = -(beta / dt) * fmax_std(0.0f, p->depth - SLOP);
                float b = bias + p->restitution_bias;
                float dl = pr->split_impulse ? -(Jv + p->restitution_bias) * p->inv_mass : -(Jv + b) * p->inv_mass;
                float lt = p->impulse;
                p->impulse = fmax_std(p->impulse + dl, 0.0f);
                dl = p->impulse - lt;
                v3 li = V(p->normal.x * dl, p->normal.y * dl, p->normal.z * dl);
                cv[b1].x -= c->im1 * li.x * c->lf1.x; cv[b1].y -= c->im1 * li.y * c->lf1.y; cv[b1].z -= c->im1 * li.z * c->lf1.z;
                cw[b1].x -= p->i1.x * c->af1.x * dl; cw[b1].y -= p->i1.y * c->af1.y * dl; cw[b1].z -= p->i1.z * c->af1.z * dl;
                cv[b2].x += c->im2 * li.x * c->lf2.x; cv[b2].y += c->im2 * li.y * c->lf2.y; cv[b2].z += c->im2 * li.z * c->lf2.z;
                cw[b2].x += p->i2.x * c->af2.x * dl; cw[b2].y += p->i2.y * c->af2.y * dl; cw[b2].z += p->i2.z * c->af2.z * dl;
                sum += p->impulse;
                if (pr->split_impulse) {
                    v3 dvs = rel_vel(sv[b1], sw[b1], sv[b2], sw[b2], p->r1, p->r2);
                    float Jvs = dvs.x * p->normal.x + dvs.y * p->normal.y + dvs.z * p->normal.z;
                    float dls = -(Jvs + bias) * p->inv_mass;
                    float lts = p->split_impulse;
                    p->split_impulse = fmax_std(p->split_impulse + dls, 0.0f);
                    dls = p->split_impulse - lts;
                    v3 ls = V(p->normal.x * dls, p->normal.y * dls, p->normal.z * dls);
                    sv[b1].x -= c->im1 * ls.x * c->lf1.x; sv[b1].y -= c->im1 * ls.y * c->lf1.y; sv[b1].z -= c->im1 * ls.z * c->lf1.z;
                    sw[b1].x -= p->i1.x * c->af1.x * dls; sw[b1].y -= p->i1.y * c->af1.y * dls; sw[b1].z -= p->i1.z * c->af1.z * dls;
                    sv[b2].x += c->im2 * ls.x * c->lf2.x; sv[b2].y += c->im2 * ls.y * c->lf2.y; sv[b2].z += c->im2 * ls.z * c->lf2.z;
                    sw[b2].x += p->i2.x * c->af2.x * dls; sw[b2].y += p->i2.y * c->af2.y * dls; sw[b2].z += p->i2.z * c->af2.z * dls;
                }
            }
            /* friction 1 */
            {
                v3 dv = rel_vel(cv[b1], cw[b1], cv[b2], cw[b2], c->r1f, c->r2f);
                float Jv = dv.x * c->fv1.x + dv.y * c->fv1.y + dv.z * c->fv1.z;
                float dl = -Jv * c->inv_f1, lim = c->friction * sum, lt = c->f1;
                c->f1 = fmax_std(-lim, fmin_std(c->f1 + dl, lim));
                dl = c->f1 - lt;
                v3 a1 = V(-c->r1ct1.x * dl, -c->r1ct1.y * dl, -c->r1ct1.z * dl);
                v3 l2 = V(c->fv1.x * dl, c->fv1.y * dl, c->fv1.z * dl);
                v3 a2 = V(c->r2ct1.x * dl, c->r2ct1.y * dl, c->r2ct1.z * dl);
                cv[b1].x -= c->im1 * l2.x * c->lf1.x; cv[b1].y -= c->im1 * l2.y * c->lf1.y; cv[b1].z -= c->im1 * l2.z * c->lf1.z;
                v3 av1 = vcmul(c->af1, m3v(c->I1, a1));
                cw[b1].x += av1.x; cw[b1].y += av1.y; cw[b1].z += av1.z;
                cv[b2].x += c->im2 * l2.x * c->lf2.x; cv[b2].y += c->im2 * l2.y * c->lf2.y; cv[b2].z += c->im2 * l2.z * c->lf2.z;
                v3 av2 = vcmul(c->af2, m3v(c->I2, a2));
                cw[b2].x += av2.x; cw[b2].y += av2.y; cw[b2].z += av2.z;
            }
            /* friction 2 */
            {
                v3 dv = rel_vel(cv[b1], cw[b1], cv[b2], cw[b2], c->r1f, c->r2f);
                float Jv = dv.x * c->fv2.x + dv.y * c->fv2.y + dv.z * c->fv2.z;
                float dl = -Jv * c->inv_f2, lim = c->friction * sum, lt = c->f2;
                c->f2 = fmax_std(-lim, fmin_std(c->f2 + dl, lim));
                dl = c->f2 - lt;
                v3 a1 = V(-c->r1ct2.x * dl, -c->r1ct2.y * dl, -c->r1ct2.z * dl);
                v3 l2 = V(c->fv2.x * dl, c->fv2.y * dl, c->fv2.z * dl);
                v3 a2 = V(c->r2ct2.x * dl, c->r2ct2.y * dl, c->r2ct2.z * dl);
                cv[b1].x -= c->im1 * l2.x * c->lf1.x; cv[b1].y -= c->im1 * l2.y * c->lf1.y; cv[b1].z -= c->im1 * l2.z * c->lf1.z;
                v3 av1 = vcmul(c->af1, m3v(c->I1, a1));
                cw[b1].x += av1.x; cw[b1].y += av1.y; cw[b1].z += av1.z;
                cv[b2].x += c->im2 * l2.x * c->lf2.x; cv[b2].y += c->im2 * l2.y * c->lf2.y; cv[b2].z += c->im2 * l2.z * c->lf2.z;
                v3 av2 = vcmul(c->af2, m3v(c->I2, a2));
                cw[b2].x += av2.x; cw[b2].y += av2.y; cw[b2].z += av2.z;
            }
            /* twist */
            {
                v3 dw = vsub(cw[b2], cw[b1]);
                float Jv = dw.x * c->normal.x + dw.y * c->normal.y + dw.z * c->normal.z;
                float dl = -Jv * c->inv_tw, lim = c->friction * sum, lt = c->ftw;
                c->ftw = fmax_std(-lim, fmin_std(c->ftw + dl, lim));
                dl = c->ftw - lt;
                v3 a2 = V(c->normal.x * dl, c->normal.y * dl, c->normal.z * dl);
                v3 av1 = vcmul(c->af1, m3v(c->I1, a2));
                cw[b1].x -= av1.x; cw[b1].y -= av1.y; cw[b1].z -= av1.z;
                v3 av2 = vcmul(c->af2, m3v(c->I2, a2));
                cw[b2].x += av2.x; cw[b2].y += av2.y; cw[b2].z += av2.z;
            }
        }
    }

    /* storeImpulses (:763-785) */
    {
        uint32_t q = 0;
        for (uint32_t k = 0; k < nm; k++) {
            DynMan* c = &man[k];
            for (int i = 0; i < c->nb; i++, q++) P->penetration_impulse[pt[q].ext] = pt[q].impulse;
            rp3dg_float4 fi; fi.x = c->f1; fi.y = c->f2; fi.z = c->ftw; fi.w = 0.0f;
            M->friction_impulse[c->ext] = fi;
            M->friction_vector1[c->ext] = S4(c->fv1);
            M->friction_vector2[c->ext] = S4(c->fv2);
        }
    }

    /* integrateRigidBodiesPositions + updateBodiesState (DynamicsSystem.cpp:44-110) */
    const float f = pr->split_impulse ? 1.0f : 0.0f;
    quat* co = (quat*)calloc(ne ? ne : 1, sizeof(quat));
    v3* cp = (v3*)calloc(ne ? ne : 1, sizeof(v3));
    for (uint32_t i = 0; i < ne; i++) {
        v3 nl = vadd(cv[i], vmul(sv[i], f)), na = vadd(cw[i], vmul(sw[i], f));
        rp3dg_float4 o = B->orientation[i];
        quat q = Q(o.x, o.y, o.z, o.w);
        cp[i] = vadd(L4(B->com_world[i]), vmul(nl, dt));
        quat d = qmul(Q(na.x, na.y, na.z, 0.0f), q);
        d = Q(0.5f * d.x, 0.5f * d.y, 0.5f * d.z, 0.5f * d.w);
        d = Q(dt * d.x, dt * d.y, dt * d.z, dt * d.w);
        co[i] = Q(q.x + d.x, q.y + d.y, q.z + d.z, q.w + d.w);
    }
    for (uint32_t i = 0; i < ne; i++) {
        B->linear_velocity[i] = S4(cv[i]);
        B->angular_velocity[i] = S4(cw[i]);
        B->com_world[i] = S4(cp[i]);
        quat q = co[i];
        float l = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        rp3dg_float4 o; o.x = q.x / l; o.y = q.y / l; o.z = q.z / l; o.w = q.w / l;
        B->orientation[i] = o;
    }
    for (uint32_t i = 0; i < ne; i++) {
        rp3dg_float4 o = B->orientation[i];
        B->position[i] = S4(vsub(cp[i], qrot(Q(o.x, o.y, o.z, o.w), L4(B->com_local[i]))));
    }
    for (uint32_t i = 0; i < Cl->n_enabled; i++) {
        int b = Cl->body[i];
        rp3dg_float4 bo = B->orientation[b], lo = Cl->local_orientation[i];
        xform t = xmul(X(L4(B->position[b]), Q(bo.x, bo.y, bo.z, bo.w)), X(L4(Cl->local_position[i]), Q(lo.x, lo.y, lo.z, lo.w)));
        Cl->world_position[i] = S4(t.p);
        rp3dg_float4 wq; wq.x = t.q.x; wq.y = t.q.y; wq.z = t.q.z; wq.w = t.q.w;
        Cl->world_orientation[i] = wq;
    }
    free(co); free(cp);
    free(cv); free(cw); free(sv); free(sw); free(man); free(pt);
    return 0;
}

/* ===================================================================== */
/* Broad phase: collider AABBs and fat AABBs (BroadPhaseSystem.cpp:       */
/* 155-185, CollisionShape.cpp:54-90, SphereShape.cpp:49-58,              */
/* DynamicAABBTree.cpp:186-214), and the overlapping-pair set             */
/* (CollisionDetectionSystem.cpp:270-343 with DynamicAABBTree.cpp:589-638) */
/* ===================================================================== */

/* CollisionShape::getLocalBounds of the shape kinds of rp3dg.h */
static void local_bounds(const rp3dg_shape* s, const float* mesh_bounds, v3* mn, v3* mx) {
    const float* p = s->params;
    switch (s->kind) {
        case RP3DG_SHAPE_SPHERE: *mn = V(-p[0], -p[0], -p[0]); *mx = V(p[0], p[0], p[0]); break;
        case RP3DG_SHAPE_CAPSULE: *mn = V(-p[0], -p[1] - p[0], -p[0]); *mx = V(p[0], p[1] + p[0], p[0]); break;
        case RP3DG_SHAPE_BOX: *mn = V(-p[0], -p[1], -p[2]); *mx = V(p[0], p[1], p[2]); break;
        default: *mn = V(mesh_bounds[0], mesh_bounds[1], mesh_bounds[2]); *mx = V(mesh_bounds[3], mesh_bounds[4], mesh_bounds[5]); break;
    }
}

int rp3do_broadphase_update(const rp3dg_shape* shapes, const float* mesh_bounds, uint32_t n, const int32_t* shape,
                            const rp3dg_float4* wpos, const rp3dg_float4* wori, const uint8_t* force,
                            rp3dg_float4* fat_min, rp3dg_float4* fat_max, uint8_t* moved) {
    for (uint32_t i = 0; i < n; i++) {
        const rp3dg_shape* s = &shapes[shape[i]];
        v3 t = L4(wpos[i]);
        v3 amin, amax;
        if (s->kind == RP3DG_SHAPE_SPHERE) {
            v3 e = V(s->params[0], s->params[0], s->params[0]);
            amin = vsub(t, e); amax = vadd(t, e);
        } else {
            v3 lmn, lmx;
            local_bounds(s, mesh_bounds ? mesh_bounds + 6 * (s->mesh < 0 ? 0 : s->mesh) : NULL, &lmn, &lmx);
            float m[9];
            q_matrix(Q(wori[i].x, wori[i].y, wori[i].z, wori[i].w), m);
            float rmin[3], rmax[3], tt[3] = {t.x, t.y, t.z}, bmin[3] = {lmn.x, lmn.y, lmn.z}, bmax[3] = {lmx.x, lmx.y, lmx.z};
            for (int a = 0; a < 3; a++) {
                rmin[a] = tt[a]; rmax[a] = tt[a];
                for (int b = 0; b < 3; b++) {
                    float e = m[3 * a + b] * bmin[b], f = m[3 * a + b] * bmax[b];
                    if (e < f) { rmin[a] += e; rmax[a] += f; }
                    else { rmin[a] += f; rmax[a] += e; }
                }
            }
            amin = V(rmin[0], rmin[1], rmin[2]); amax = V(rmax[0], rmax[1], rmax[2]);
        }
        v3 fmn = L4(fat_min[i]), fmx = L4(fat_max[i]);
        int inside = fmn.x <= amin.x && fmn.y <= amin.y && fmn.z <= amin.z &&
                     fmx.x >= amax.x && fmx.y >= amax.y && fmx.z >= amax.z;
        if ((!force || !force[i]) && inside) { moved[i] = 0; continue; }
        v3 ext = vsub(amax, amin);
        v3 gap = vmul(vmul(ext, 0.08f), 0.5f);   /* DYNAMIC_TREE_FAT_AABB_INFLATE_PERCENTAGE (configuration.h:131) */
        fat_min[i] = S4(vsub(amin, gap));
        fat_max[i] = S4(vadd(amax, gap));
        moved[i] = 1;
    }
    return 0;
}

/* All pairs (i < j) whose fat AABBs overlap (AABB::testCollision, inclusive),
 * of different bodies and the same group, passing the category / mask
 * filter.  Writes up to cap pairs, returns the count (may exceed cap). */
long rp3do_broadphase_pairs(uint32_t n, const rp3dg_float4* fat_min, const rp3dg_float4* fat_max, const int32_t* body,
                            const int32_t* group, const uint16_t* category, const uint16_t* mask, int32_t* pairs,
                            long cap) {
    long count = 0;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = i + 1; j < n; j++) {
            if (group && group[i] != group[j]) continue;
            const rp3dg_float4 a0 = fat_min[i], a1 = fat_max[i], b0 = fat_min[j], b1 = fat_max[j];
            if (a1.x < b0.x || b1.x < a0.x) continue;
            if (a1.y < b0.y || b1.y < a0.y) continue;
            if (a1.z < b0.z || b1.z < a0.z) continue;
            if (body[i] == body[j]) continue;
            if (category && mask && (!(mask[i] & category[j]) || !(category[i] & mask[j]))) continue;
            if (count < cap) { pairs[2 * count] = (int32_t)i; pairs[2 * count + 1] = (int32_t)j; }
            count++;
        }
    return count;
}
