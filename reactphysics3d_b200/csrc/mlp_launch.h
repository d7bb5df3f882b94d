// Launch interface of the separating-axis MLP kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rp3dg.h"
#include "rp3dg_internal.h"

namespace rp3dg {

struct MlpPacked;

constexpr int MLP_IN = 24, MLP_H = 64, MLP_OUT = 16, MLP_KPAD = 32;
constexpr int MLP_NO_PROPOSAL = 15;
// parameter vector layout (fp32 masters): w1[24][64] b1[64] w2[64][64] b2[64] w3[64][16] b3[16]
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_IN * MLP_H;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_H * MLP_OUT;
constexpr int MLP_NPARAMS = MLP_OFF_B3 + MLP_OUT;  // 6800

// floats per sample of training scratch: h1[64] h2[64] dh1[64] dh2[64] dz[16]
constexpr int MLP_SCRATCH_ROW = 272;

struct MlpPairArgs {
    uint32_t n;
    uint32_t nb_shapes;
    const rp3dg_shape* shapes;
    const int32_t* shape1;
    const int32_t* shape2;
    const float4* pos1;
    const float4* rot1;
    const float4* pos2;
    const float4* rot2;
    const uint32_t* mesh_words;
    const BoxTables* box;
};

void upload_mlp_box_tables(const BoxTables& t, cudaStream_t s);
cudaError_t launch_axis_features(const MlpPairArgs& a, float* feat, cudaStream_t s);
cudaError_t launch_axis_labels(const MlpPairArgs& a, const uint8_t* colliding, const rp3dg_lastframe* cache,
                               uint8_t* labels, cudaStream_t s);
cudaError_t launch_mlp_grads(const float* params, const float* x, const uint8_t* y, uint32_t n, float* scratch,
                             float* grads, float* loss_sum, cudaStream_t s);
cudaError_t launch_mlp_adam(float* params, const float* grads, float* m, float* v, float lr, int step, cudaStream_t s);
cudaError_t launch_mlp_pack(const float* params, MlpPacked* out, cudaStream_t s);
// Largest batch of rp3dg_axis_mlp_grads_noalloc (its scratch is a fixed array).
constexpr uint32_t MLP_NOALLOC_MAX_SAMPLES = 4096;
cudaError_t launch_mlp_grads_noalloc(const float* params, const float* x, const uint8_t* y, uint32_t n, float* grads,
                                     float* loss_host, cudaStream_t s);
cudaError_t launch_mlp_predict(const MlpPacked* w, const float* x, uint32_t n, uint8_t* cls, int num_sms, cudaStream_t s);

}  // namespace rp3dg
