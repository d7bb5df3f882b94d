// Learned separating-axis proposal for convex polyhedron pairs (no
// counterpart in the reference engine).
//
// A small MLP (24 -> 64 -> 64 -> 16, ReLU, bf16 weights, fp32 accumulation)
// maps the relative pose of a pair to one of 16 classes:
//   0..2   a face of polyhedron 1 whose normal is local axis x / y / z (box)
//   3..5   a face of polyhedron 2 whose normal is local axis x / y / z (box)
//   6..14  an edge of polyhedron 1 along axis a = (c-6)/3 crossed with an edge
//          of polyhedron 2 along axis b = (c-6)%3 (box-box)
//   15     no proposal (colliding, or a separating feature outside 0..14)
// A proposal is used only where the reference would run its full SAT, and it
// only counts when the reference's own exact test of that feature
// (testSingleFaceDirectionPolyhedronVsPolyhedron, SATAlgorithm.cpp:1087-1110;
// testEdgesBuildMinkowskiFace + computeDistanceBetweenEdges, :1146-1172 and
// :1040-1083) finds a separating axis.  A separating axis among the SAT
// candidates means the reference's full SAT also returns "no contact", so the
// contacts are unchanged; only the cached axis may name a different (also
// separating) feature than the reference's first one.
#pragma once
#include <cuda_bf16.h>

#include "mlp_launch.h"
#include "narrowphase.cuh"

namespace rp3dg {


// Weights packed as mma.m16n8k16 B fragments (bf16 pairs): for layer L with
// KS k-steps and NT n-tiles, entry ((ks * NT + nt) * 32 + lane) holds
// {W[16ks + 2t .. +1][8nt + g], W[16ks + 8 + 2t .. +1][8nt + g]}, g = lane/4,
// t = lane%4.  Followed by the fp32 biases.
constexpr int MLP_FRAG_L1 = (MLP_KPAD / 16) * (MLP_H / 8) * 32;   // uint2 entries
constexpr int MLP_FRAG_L2 = (MLP_H / 16) * (MLP_H / 8) * 32;
constexpr int MLP_FRAG_L3 = (MLP_H / 16) * (MLP_OUT / 8) * 32;
struct MlpPacked {
    uint2 l1[MLP_FRAG_L1];
    uint2 l2[MLP_FRAG_L2];
    uint2 l3[MLP_FRAG_L3];
    float b1[MLP_H], b2[MLP_H], b3[MLP_OUT];
};

// Rotation matrix of a quaternion (row-major), the usual expansion.
RD void quat_matrix(quat q, float m[9]) {
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    m[0] = 1.0f - 2.0f * (y * y + z * z); m[1] = 2.0f * (x * y - w * z);        m[2] = 2.0f * (x * z + w * y);
    m[3] = 2.0f * (x * y + w * z);        m[4] = 1.0f - 2.0f * (x * x + z * z); m[5] = 2.0f * (y * z - w * x);
    m[6] = 2.0f * (x * z - w * y);        m[7] = 2.0f * (y * z + w * x);        m[8] = 1.0f - 2.0f * (x * x + y * y);
}

// Half-extents of a polyhedron's local bounds (box: its half-extents; mesh:
// the largest |coordinate| over its scaled vertices).
RD v3 poly_half_extents(const BoxPoly& b) { return b.he; }
RD v3 poly_half_extents(const MeshPoly& m) {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    const uint32_t nv = m.h->nv;
    for (uint32_t i = 0; i < nv; i++) {
        const v3 v = m.vertex(i);
        x = fmaxf(x, fabsf(v.x)); y = fmaxf(y, fabsf(v.y)); z = fmaxf(z, fabsf(v.z));
    }
    return V(x, y, z);
}

// The 24 input features of a pair (shape 1 pose relative to shape 2).
template <class P1, class P2>
RD void axis_features(const xform& t1, const xform& t2, const P1& p1, const P2& p2, bool mesh1, float f[MLP_IN]) {
    const xform p1to2 = xmul(xinv(t2), t1);
    const xform p2to1 = xinv(p1to2);
    quat_matrix(p1to2.q, f);
    f[9] = p1to2.p.x; f[10] = p1to2.p.y; f[11] = p1to2.p.z;
    const v3 h1 = poly_half_extents(p1), h2 = poly_half_extents(p2);
    f[12] = h1.x; f[13] = h1.y; f[14] = h1.z;
    f[15] = h2.x; f[16] = h2.y; f[17] = h2.z;
    f[18] = p2to1.p.x; f[19] = p2to1.p.y; f[20] = p2to1.p.z;
    const float d = vlen(p1to2.p);
    f[21] = d;
    f[22] = d / (vlen(h1) + vlen(h2));
    f[23] = mesh1 ? 1.0f : 0.0f;
}

// Box face axis: faces 1/3 -> x, 5/4 -> y, 0/2 -> z (BoxShape.h:211-225).
RD uint32_t box_face_axis(uint32_t f) { return f == 1 || f == 3 ? 0u : (f == 4 || f == 5 ? 1u : 2u); }

// Training label of a pair from the outcome of the plain SAT: colliding ->
// 15; otherwise the class of the separating feature the SAT cached, or 15
// when that feature is not one of the 15 candidates (a mesh face or edge).
RD uint32_t axis_label(bool colliding, const LastFrame& lf, bool box1, bool box2, const BoxTables* bt) {
    if (colliding) return MLP_NO_PROPOSAL;
    if (lf.has(RP3DG_LF_SAT_FACE_POLY1)) return box1 ? box_face_axis(lf.sat_face) : MLP_NO_PROPOSAL;
    if (lf.has(RP3DG_LF_SAT_FACE_POLY2)) return box2 ? 3u + box_face_axis(lf.sat_face) : MLP_NO_PROPOSAL;
    if (!(box1 && box2)) return MLP_NO_PROPOSAL;
    const uint32_t a = bt->gauss[lf.sat_e1][0] & 3u, b = bt->gauss[lf.sat_e2][0] & 3u;
    return 6u + 3u * a + b;
}

// ---------------------------------------------------------------------------
// warp-level bf16 tensor-core inference for 32 pairs (one per lane)
// ---------------------------------------------------------------------------
RD uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

RD void mma_bf16_16816(float c[4], const uint32_t a[4], uint2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// x: the tile's features in shared memory, [32][MLP_KPAD] fp32 (row = lane's
// pair, columns 24..31 zero).  Returns the arg-max class of the caller's pair
// (lane); all 32 lanes must call.
RD uint32_t mlp_infer_tile(const float (*x)[MLP_KPAD], const MlpPacked& w, int lane, uint32_t* cls) {
    const int g = lane >> 2, t = lane & 3;
    uint32_t a[2][MLP_H / 16][4];  // bf16 A fragments of the current layer input (2 m-tiles)
    // layer-1 input fragments straight from the feature rows
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
#pragma unroll
        for (int ks = 0; ks < MLP_KPAD / 16; ks++) {
            const float* r0 = x[16 * mt + g];
            const float* r1 = x[16 * mt + g + 8];
            const int c = 16 * ks + 2 * t;
            a[mt][ks][0] = pack_bf16x2(r0[c], r0[c + 1]);
            a[mt][ks][1] = pack_bf16x2(r1[c], r1[c + 1]);
            a[mt][ks][2] = pack_bf16x2(r0[c + 8], r0[c + 9]);
            a[mt][ks][3] = pack_bf16x2(r1[c + 8], r1[c + 9]);
        }
    }
    float acc[2][MLP_H / 8][4];
    // layer 1: [32 x 32] x [32 x 64]
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < MLP_H / 8; nt++) {
            acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.0f;
#pragma unroll
            for (int ks = 0; ks < MLP_KPAD / 16; ks++) mma_bf16_16816(acc[mt][nt], a[mt][ks], w.l1[(ks * (MLP_H / 8) + nt) * 32 + lane]);
        }
    // bias + ReLU, re-packed as the next layer's A fragments
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int ks = 0; ks < MLP_H / 16; ks++) {
            float v[8];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int nt = 2 * ks + h, col = 8 * nt + 2 * t;
                v[4 * h + 0] = fmaxf(acc[mt][nt][0] + w.b1[col], 0.0f);
                v[4 * h + 1] = fmaxf(acc[mt][nt][1] + w.b1[col + 1], 0.0f);
                v[4 * h + 2] = fmaxf(acc[mt][nt][2] + w.b1[col], 0.0f);
                v[4 * h + 3] = fmaxf(acc[mt][nt][3] + w.b1[col + 1], 0.0f);
            }
            a[mt][ks][0] = pack_bf16x2(v[0], v[1]);
            a[mt][ks][1] = pack_bf16x2(v[2], v[3]);
            a[mt][ks][2] = pack_bf16x2(v[4], v[5]);
            a[mt][ks][3] = pack_bf16x2(v[6], v[7]);
        }
    // layer 2: [32 x 64] x [64 x 64]
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < MLP_H / 8; nt++) {
            acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.0f;
#pragma unroll
            for (int ks = 0; ks < MLP_H / 16; ks++) mma_bf16_16816(acc[mt][nt], a[mt][ks], w.l2[(ks * (MLP_H / 8) + nt) * 32 + lane]);
        }
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int ks = 0; ks < MLP_H / 16; ks++) {
            float v[8];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int nt = 2 * ks + h, col = 8 * nt + 2 * t;
                v[4 * h + 0] = fmaxf(acc[mt][nt][0] + w.b2[col], 0.0f);
                v[4 * h + 1] = fmaxf(acc[mt][nt][1] + w.b2[col + 1], 0.0f);
                v[4 * h + 2] = fmaxf(acc[mt][nt][2] + w.b2[col], 0.0f);
                v[4 * h + 3] = fmaxf(acc[mt][nt][3] + w.b2[col + 1], 0.0f);
            }
            a[mt][ks][0] = pack_bf16x2(v[0], v[1]);
            a[mt][ks][1] = pack_bf16x2(v[2], v[3]);
            a[mt][ks][2] = pack_bf16x2(v[4], v[5]);
            a[mt][ks][3] = pack_bf16x2(v[6], v[7]);
        }
    // layer 3: [32 x 64] x [64 x 16] -> logits
    float z[2][2][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 2; nt++) {
            z[mt][nt][0] = z[mt][nt][1] = z[mt][nt][2] = z[mt][nt][3] = 0.0f;
#pragma unroll
            for (int ks = 0; ks < MLP_H / 16; ks++) mma_bf16_16816(z[mt][nt], a[mt][ks], w.l3[(ks * (MLP_OUT / 8) + nt) * 32 + lane]);
        }
    // arg-max of every row: each lane holds 4 logits of rows g and g+8 (per m-tile)
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int half = 0; half < 2; half++) {
            float best = -FLT_MAX;
            uint32_t bi = 0;
#pragma unroll
            for (int nt = 0; nt < 2; nt++)
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int col = 8 * nt + 2 * t + e;
                    const float v = z[mt][nt][2 * half + e] + w.b3[col];
                    if (v > best) { best = v; bi = uint32_t(col); }
                }
#pragma unroll
            for (int o = 1; o < 4; o <<= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, best, o);
                const uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (t == 0) cls[16 * mt + g + 8 * half] = bi;
        }
    __syncwarp();
    const uint32_t mine = cls[lane];
    __syncwarp();
    return mine;
}

}  // namespace rp3dg
