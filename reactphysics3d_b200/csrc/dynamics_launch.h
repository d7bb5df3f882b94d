// Launch interface of the dynamics-stage kernels (dynamics.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"

namespace rp3dg {

// Per-manifold solver record (ContactManifoldSolver, ContactSolverSystem.h:
// 153-260) and per-point record (ContactPointSolver, :85-135), in device
// scratch; one thread touches a record at a time.
struct DynManifoldRec {
    int32_t b1, b2, nb, pstart;
    float im1, im2, friction, fixed_mask;   // fixed_mask: bit0 body 1, bit1 body 2 never written
    float lf1[3], lf2[3], alf1[3], alf2[3];
    float I1[9], I2[9];
    float normal[3];
    float r1f[3], r2f[3];
    float fv1[3], fv2[3];
    float ofv1[3], ofv2[3];
    float r1ct1[3], r1ct2[3], r2ct1[3], r2ct2[3];
    float inv_f1, inv_f2, inv_tw;
    float f1, f2, ftw;
    float pad[2];
};

struct DynPointRec {
    float r1[3], depth;
    float r2[3], inv_mass;
    float normal[3], restitution_bias;
    float i1[3], impulse;
    float i2[3], split_impulse;
    uint32_t resting, pad[3];
};

struct DynArgs {
    // params
    float dt, gx, gy, gz;
    int32_t gravity_enabled, iterations, split;
    float restitution_threshold;
    // bodies
    uint32_t nb, nb_enabled;
    float4 *position, *orientation, *com_world;
    const float4* com_local;
    float4 *lin_vel, *ang_vel;
    const float4 *force, *torque, *iil;
    float4* iiw;
    const float4 *mass, *llock, *alock;
    const uint8_t* gravity;
    // colliders
    uint32_t nc, nc_enabled;
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
};

// Launches the five kernels in order on stream s; *launches += 5.
cudaError_t launch_dynamics(const DynArgs& a, cudaStream_t s, uint64_t* launches);

}  // namespace rp3dg
