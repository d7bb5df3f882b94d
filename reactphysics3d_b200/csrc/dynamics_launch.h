// Launch interface of the dynamics-stage kernels (dynamics.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"

namespace rp3dg {

// Per-manifold solver record (the data of ContactManifoldSolver,
// ContactSolverSystem.h:153-260) and per-point record (ContactPointSolver,
// :85-135) in device scratch, as rows of float4 so that the solver loads each
// with one 16-byte access.  q[] is written once by the manifold kernel;
// mut holds what the passes update.
enum DynManifoldRow {
    DQ_IDS = 0,     // body1, body2, number of points, first point (int bits)
    DQ_MASS,        // inverse mass 1, inverse mass 2, friction coefficient, fixed mask (bit0 body1, bit1 body2)
    DQ_LF1, DQ_LF2, DQ_AF1, DQ_AF2,   // linear / angular lock factors
    DQ_I1, DQ_I2 = DQ_I1 + 3,          // world inverse inertia rows
    DQ_N = DQ_I2 + 3,                  // normal, inverse twist friction mass
    DQ_R1F, DQ_R2F,                    // friction point arms, inverse friction 1 / 2 masses
    DQ_FV1, DQ_FV2,                    // friction vectors
    DQ_R1CT1, DQ_R1CT2, DQ_R2CT1, DQ_R2CT2,
    DQ_OFV1, DQ_OFV2,                  // previous friction vectors (warm start)
    DQ_ROWS
};
struct __align__(16) DynManifoldRec {
    float4 q[DQ_ROWS];
    float4 mut;   // friction 1, friction 2, twist impulses; w: scheduling level
};

enum DynPointRow { DP_R1 = 0, DP_R2, DP_N, DP_I1, DP_I2, DP_ROWS };  // (r1, depth), (r2, inverse mass), (n, restitution bias)
struct __align__(16) DynPointRec {
    float4 q[DP_ROWS];
    float4 mut;   // penetration impulse, split impulse, resting (1 / 0)
};

// Statistics of one dynamics stage for a solver comparison: the velocity
// constraint residual over the contact points after the last iteration (per
// point |n . dv| when its accumulated impulse is positive, else the
// approaching speed max(0, -n . dv)), and the bodies' energies after the
// stage (kinetic: translational + rotational; potential: -m g . x).
struct SolverStats {
    double residual_sq_sum;
    double kinetic;
    double potential;
    uint32_t residual_max_bits;   // float bits of the largest residual (non-negative)
    uint32_t points;
    uint32_t colors;              // graph-coloured solver: colours and colouring rounds
    uint32_t rounds;
};

// Scratch of the graph-coloured solver (sized by the caller).
struct ColorScratch {
    uint32_t* start;     // nb + 1: first adjacency entry of each body
    uint32_t* fill;      // nb
    uint32_t* adj;       // 2 nm: manifolds of each movable body
    uint8_t* color;      // nm
    uint8_t* tent;       // nm
    uint32_t* count;     // COLOR_MAX + 2: manifolds per colour, then [COLOR_MAX] remaining, [COLOR_MAX + 1] spare
    uint32_t* offset;    // COLOR_MAX
    uint32_t* order;     // nm: manifolds sorted by colour
};
constexpr uint32_t COLOR_MAX = 128;

// Per-joint record (joints.cuh): constant rows set on creation (type and
// flags, local anchors, local hinge / slider axes, inverse initial
// orientation difference, limits / motor parameters), accumulated impulses
// and limit state carried from step to step, and the rows initBeforeSolve
// computes.
enum JointRow {
    JR_HDR = 0,     // x type (RP3DG_JOINT_*), y flags (int bits)
    JR_LA1, JR_LA2, // local anchor points
    JR_AX1, JR_AX2, // hinge: local axes; slider: local axis of body 1 (AX1)
    JR_QINV,        // hinge, fixed, slider: inverse initial orientation difference (quaternion)
    JR_PARAM,       // x cone half angle, y lower limit, z upper limit, w motor speed
    JR_PARAM2,      // x max motor torque (hinge) / force (slider)
    JR_IMP,         // ball-and-socket impulse / hinge, fixed translation impulse /
                    // slider: translation impulse x, y, lower-limit impulse, upper-limit impulse
    JR_IMP2,        // hinge: rotation impulse x, y, lower-limit impulse, upper-limit impulse;
                    // fixed, slider: rotation impulse
    JR_STATE,       // ball-and-socket: cone impulse, cone violated;
                    // hinge, slider: lower / upper violated, motor impulse
    JR_R1, JR_R2,
    JR_I1, JR_I2 = JR_I1 + 3, JR_K = JR_I2 + 3, JR_ACB = JR_K + 3,
    JR_A1,          // hinge / slider axis in world space
    JR_B2A1, JR_C2A1,
    JR_KROT,        // 2x2 inverse mass: hinge rotation, slider translation
    JR_MISC,        // x inverse mass of the limits (and of the hinge motor), y slider motor inverse mass
    JR_KR3,         // fixed, slider: 3x3 rotation inverse mass (3 rows)
    JR_N1 = JR_KR3 + 3, JR_N2,             // slider: the two axes orthogonal to the slider axis
    JR_R2N1, JR_R2N2, JR_R2A,              // slider: r2 x n1, r2 x n2, r2 x axis
    JR_R1N1, JR_R1N2, JR_R1A,              // slider: (r1 + u) x n1, x n2, x axis
    JR_ROWS
};
enum JointFlags { JF_CONE = 1, JF_LIMIT = 2, JF_MOTOR = 4 };
struct __align__(16) JointRec {
    float4 q[JR_ROWS];
};

// Kernel 3b stages an island's schedule and its movable bodies' velocities
// in the shared memory of the warp that solves it, when they fit.
constexpr uint32_t STAGE_BODIES = 256;
constexpr uint32_t STAGE_MANIFOLDS = 512;
constexpr int LARGE_WARPS = 3;                 // warps per CTA of kernel 3b (2 CTAs per SM)
constexpr size_t LARGE_WARP_SMEM = 34816;      // bytes of shared memory per warp

struct DynArgs {
    // params
    float dt, gx, gy, gz;
    int32_t gravity_enabled, iterations, split;
    float restitution_threshold;
    // bodies
    uint32_t nb, nb_enabled;
    const uint8_t* b_enabled;   // per-row enabled flag, or null: rows [0, nb_enabled)
    float4 *position, *orientation, *com_world;
    const float4* com_local;
    float4 *lin_vel, *ang_vel;
    const float4 *force, *torque, *iil;
    float4* iiw;
    const float4 *mass, *llock, *alock;
    const uint8_t* gravity;
    // colliders
    uint32_t nc, nc_enabled;
    const uint8_t* c_enabled;   // per-row enabled flag, or null: rows [0, nc_enabled)
    const int32_t* c_body;
    const float4 *c_lpos, *c_lori;
    float4 *c_wpos, *c_wori;
    const float4* c_mat;
    // manifolds / points / islands
    uint32_t nm, np, ni;
    const int4* m_ids;
    const uint32_t* m_pstart;
    const uint8_t* m_npts;
    float4 *m_fv1, *m_fv2, *m_fimp;
    const float4 *p_nd, *p_l1, *p_l2;
    float* p_impulse;
    uint8_t* p_resting;
    const uint32_t *i_start, *i_count;
    // error bits (bit 2: an index or range of the input is out of bounds;
    // the offending manifold, island or collider is skipped)
    uint32_t* error;
    // scratch
    float4 *cv, *cw, *sv, *sw;
    DynManifoldRec* mrec;
    DynPointRec* prec;
    uint32_t* level;       // nm: level starts per island (scratch)
    uint32_t* order;       // nm: island manifolds sorted by level (scratch)
    uint32_t* body_level;  // nb: last level of each movable body (scratch)
    int32_t* body_slot;    // nb: shared-memory slot of each movable body (scratch)
    uint32_t* counters;    // [0] big islands queued (front of large_list), [1] islands taken, [2] others queued (back),
                           // [3] giant islands queued, [4] giant islands taken,
                           // [5] streamed islands queued (back of giant_list), [6] streamed islands taken
    uint32_t* large_list;  // ni: queued islands
    uint32_t* giant_list;  // ni: islands for kernel 3c
    uint32_t large_ctas;   // grid of kernel 3b (persistent)
    uint32_t small_max;    // islands of up to this many manifolds: one thread each (kernel 3a)
    uint32_t giant_min;    // islands above this many manifolds: one CTA each (kernel 3c)
    // joints (nj = 0: none).  j_list holds this step's enabled joints island
    // by island, each island's ball-and-socket, fixed, hinge then slider
    // joints, each type in component order: record index, body 1 row, body 2 row, bit 0 / bit 1 =
    // body 1 / body 2 dynamic.  Islands with joints (i_jcount > 0) are solved
    // by kernel 3d; after the position integration kernel 4b runs the
    // position correction of their joints and updates their bodies' state.
    uint32_t nj;
    const int4* j_list;
    JointRec* j_rec;
    const uint32_t* i_jstart;
    const uint32_t* i_jcount;
    uint32_t nji;               // islands with joints
    const uint32_t* ji_island;  // their island indices
    const uint32_t* ji_bstart;  // and their enabled bodies' rows: ji_rows[ji_bstart[k] .. + ji_bcount[k])
    const uint32_t* ji_bcount;
    const int32_t* ji_rows;
    float4* xc;                 // constrained positions (centres of mass), all rows, kept between steps
    float4* qc;                 // constrained orientations, all rows
    int32_t position_iterations;
    uint32_t giant_ctas;   // grid of kernel 3c (persistent, one warp per CTA)
    uint32_t giant_smem;   // dynamic shared memory of a kernel-3c CTA (0: kernel 3c off)
    // graph-coloured solver (not the drop-in: see launch_dynamics) and the
    // solver statistics of the stage (either solver), when set
    int32_t colored;
    struct SolverStats* stats;
    ColorScratch* color;
};

// The joint part of a dynamics stage (see DynArgs).
struct DynJoints {
    uint32_t nj;
    const int4* j_list;
    JointRec* j_rec;
    const uint32_t *i_jstart, *i_jcount;
    uint32_t nji;
    const uint32_t *ji_island, *ji_bstart, *ji_bcount;
    const int32_t* ji_rows;
    float4 *xc, *qc;
    int32_t position_iterations;
};

// Scheduling of the islands over the kernels (results do not depend on it):
// thread-per-island limit, one-CTA-per-island threshold and persistent CTAs
// per SM of the warp-per-island kernel.
struct DynTuning {
    uint32_t small_max = 8, giant_min = 256, large_per_sm = 2;
};

// Solver choice of a dynamics stage: the exact-order solver (the drop-in) or
// the graph-coloured one, and where the stage's statistics go (device, or
// null for none).
struct DynSolver {
    int colored = 0;
    SolverStats* stats = nullptr;
};

// Launches the kernels in order on stream s; *launches counts them.
cudaError_t launch_dynamics(const DynArgs& a, cudaStream_t s, uint64_t* launches);

}  // namespace rp3dg
