// Launch interface of the debug-rendering kernels (debug.cu): the lines and
// triangles of DebugRenderer (src/utils/DebugRenderer.cpp) for a world's
// colliders and contact points, written into device arrays.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"
#include "rp3dg_internal.h"

namespace rp3dg {

// DebugRenderer constants (DebugRenderer.h:149-161): sphere tessellation and
// the default lengths
constexpr int DEBUG_SECTORS = 18;
constexpr int DEBUG_STACKS = 10;
// cos / sin of the stack angles (i = 0..10: PI/2 - i * PI/10) and of the
// sector angles (j = 0..18: j * 2 PI/18), computed on the host in float
// exactly as the reference computes them (std::cos / std::sin of floats)
struct DebugTrig {
    float stack_cos[DEBUG_STACKS + 1], stack_sin[DEBUG_STACKS + 1];
    float sector_cos[DEBUG_SECTORS + 1], sector_sin[DEBUG_SECTORS + 1];
};
void make_debug_trig(DebugTrig* t);

// Primitives of one collider: its device row, shape-table index and where
// its lines and triangles start.
struct DebugJob {
    int32_t row, shape;
    uint32_t line, tri;
};

struct DebugArgs {
    uint32_t items;                    // RP3DG_DEBUG_* bits
    // colliders
    uint32_t n_jobs;
    const DebugJob* jobs;
    const float4 *wpos, *wori, *fmin, *fmax;
    const rp3dg_shape* shapes;
    const float4* bounds;              // 2 per shape: local bounds min, max
    const uint32_t* mesh_words;
    const HfDesc* hf;
    const CmDesc* cm;
    // contact points: x collider-1 row in the snapshot taken before the
    // step's integration, y packed point index, z first line, w first triangle
    uint32_t n_points;
    const int4* points;
    const float4 *snap_wpos, *snap_wori;
    const float4 *nd, *l1;
    // outputs
    rp3dg_debug_line* lines;
    rp3dg_debug_triangle* tris;
    DebugTrig trig;
};

// Number of lines and triangles one collider adds (host side, same rules as
// the kernels): kind, mesh face vertex counts (convex mesh), height-field
// size, concave mesh vertices and triangles.
void debug_collider_counts(uint32_t items, int kind, const uint32_t* face_counts, uint32_t nfaces, uint32_t hf_cols,
                           uint32_t hf_rows, uint32_t cm_vertices, uint32_t cm_triangles, uint32_t* lines,
                           uint32_t* tris);
constexpr uint32_t DEBUG_SPHERE_TRIS = 324;   // 18 x (9 + 9)

cudaError_t launch_debug(const DebugArgs& a, cudaStream_t s);

}  // namespace rp3dg
