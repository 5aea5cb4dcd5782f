// mlp.h — model buffers of the learned coarse-grid PME correction (mlp.cu,
// learned.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "engine.h"

namespace lima {

constexpr int MLP_IN = 68;        // coarse force (3) + charge (1) + descriptor (64)
constexpr int MLP_KIN = 80;       // input width padded to a multiple of 16
constexpr int MLP_HID = 128;
constexpr int MLP_OUT = 3;
constexpr int MLP_K[4] = {MLP_KIN, 128, 128, 128};
constexpr int MLP_N[4] = {128, 128, 128, 8};
constexpr int MLP_CHUNK = 512;    // rows per weight-gradient partial
constexpr int DESC_RADIAL = 16;   // Gaussian centres over [0, DESC_CUT]
constexpr float DESC_CUT = 0.8f;  // [nm]
constexpr float DESC_WIDTH = 0.05f;

// parameter vector layout shared by get/set weights and the gradient check:
// W1[80][128] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] W4[128][8] b4[8]
constexpr int MLP_NPARAM = 80 * 128 + 128 + 2 * (128 * 128 + 128) + 128 * 8 + 8;
constexpr int MLP_NSTATE = MLP_NPARAM + 2 * MLP_IN + 1;   // + input mean, input std, output scale

struct MlpModel {
    float* w[4] = {};             // FP32 masters W[K][N]
    float* b[4] = {};
    float *mw[4] = {}, *vw[4] = {}, *mb[4] = {}, *vb[4] = {};   // Adam moments
    float *gw[4] = {}, *gb[4] = {};                             // gradients
    __nv_bfloat16* wb[4] = {};    // BF16 W[K][ldw] (ldw = N, 16 for the last layer)
    __nv_bfloat16* wtb[4] = {};   // BF16 WT[N][K]
    __nv_bfloat16* tmp[2] = {};   // inference ping-pong activations [rows][128]
    float* part = nullptr;        // weight-gradient partials
    float* bpart = nullptr;       // bias-gradient partials
    int max_rows = 0;             // rows the training buffers hold
    int* tc_err = nullptr;        // set when a bounded wait of the tcgen05 kernel gave up
    bool use_tc = true;           // inference on tcgen05 (else warp-level mma.sync)
    int adam_step = 0;
    float in_mean[MLP_IN] = {}, in_std[MLP_IN] = {};   // input normalisation
    float out_scale = 1.f;                             // residual scale [J/mol/nm]
};

struct MlpActs {                  // training activations for one batch
    __nv_bfloat16* z[3] = {};     // pre-activations [rows][128]
    __nv_bfloat16* h[3] = {};     // SiLU outputs [rows][128]
    __nv_bfloat16* dz[3] = {};    // gradients of the pre-activations
    __nv_bfloat16* dz4 = nullptr; // output gradient [rows][16]
    float* y = nullptr;           // outputs [rows][8]
};

void mlp_sync_bf16(MlpModel& m, cudaStream_t s);
// inference of all four layers in one persistent kernel, inputs normalised on the fly
int mlp_infer(const MlpModel& m, int rows, const float* feat, const float* mean, const float* inv_std, float* Y,
              cudaStream_t s);
// the same on the tcgen05 tensor cores (TMEM accumulators); *err is set if a
// bounded wait gave up
int mlp_infer_tc(const MlpModel& m, int rows, const float* feat, const float* mean, const float* inv_std, float* Y,
                 int* err, cudaStream_t s, int withhold = 0);
int mlp_forward(const MlpModel& m, int rows, const __nv_bfloat16* X, MlpActs* acts, float* Y, cudaStream_t s);
int mlp_train_step(MlpModel& m, int rows, const __nv_bfloat16* X, const float* T, MlpActs& a, float lr,
                   double* d_loss, cudaStream_t s);

// learned.cu
int launch_descriptor(const DevState& st, const long long* fc /*3 x n_slots*/, float* feat, cudaStream_t s);
int launch_mlp_input(const DevState& st, const float* feat, const float* mean, const float* inv_std,
                     __nv_bfloat16* X, cudaStream_t s);
int launch_mlp_apply(const DevState& st, const long long* fc, const float* Y, float out_scale, cudaStream_t s);
int launch_collect(const DevState& st, const float* feat, const long long* fc, const long long* ff,
                   float* rows_feat, float* rows_target, cudaStream_t s);
int launch_gather_batch(const float* rows_feat, const float* rows_target, const int* idx, int n,
                        const float* mean, const float* inv_std, float out_inv_scale, __nv_bfloat16* X, float* T,
                        cudaStream_t s);
int launch_pred_error(const DevState& st, const long long* fc, const float* Y, float scale, const long long* ff,
                      double* sums, cudaStream_t s);
int launch_add_forces(const DevState& st, const long long* src, cudaStream_t s);
int launch_rows_to_bf16(int n, const float* x, __nv_bfloat16* X, cudaStream_t s);

}  // namespace lima
