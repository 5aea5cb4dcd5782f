// learned.cu — per-atom features and force plumbing of the learned coarse-grid
// PME correction.  The reference has no learned component; this file only
// feeds mlp.cu and adds its output to the engine's fixed-point forces.
//
// Feature row of one atom (MLP_IN = 68 floats, slot order):
//   [0..2]  reciprocal force from the coarse grid [J/mol/nm]
//   [3]     charge [kC/mol]
//   [4..67] descriptor: 4 channels x 16 Gaussians of the neighbour distance,
//           G_k(r) = exp(-(r - mu_k)^2 / (2 w^2)), mu_k = k * 0.8/15 nm, w = 0.05 nm,
//           summed over neighbours j within 0.8 nm (minimum image) with weights
//             channel 0: q_j fc(r)            channel 1..3: q_j fc(r) d_x,y,z / r
//           q_j in elementary charges, fc(r) = (cos(pi r / 0.8) + 1) / 2,
//           d = r_j - r_i.  Index 4 + 16 * channel + k.
// The network's output is the residual (full-grid minus coarse-grid force) in
// units of a per-model scale; the training targets are collected per atom in
// the original atom order so that frames line up row by row.
#include <cuda_bf16.h>

#include "engine.h"
#include "mlp.h"

namespace lima {

namespace {
constexpr float kE = 96.48533212331002f;          // elementary charge [kC/mol]
constexpr float kDescReach = DESC_CUT + 0.1f;     // column window: cutoff + drift since binning
inline unsigned nblk(long long n, int tb) { return (unsigned)((n + tb - 1) / tb); }
}  // namespace

__device__ __forceinline__ int wrap_col(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// the 16 Gaussians at distance r from the nearest centre outwards: three
// exponentials and a constant ratio step (exp(-B) between neighbouring ratios)
__device__ __forceinline__ void radial16(float r, float* g) {
    constexpr float d = DESC_CUT / (DESC_RADIAL - 1);
    constexpr float i2w2 = 1.f / (2.f * DESC_WIDTH * DESC_WIDTH);
    constexpr float B = 2.f * d * d * i2w2;
    const float F = __expf(-B);
    const int kc = min(DESC_RADIAL - 1, max(0, __float2int_rn(r / d)));
    const float dc = r - kc * d;
    const float A = (2.f * d * r - d * d) * i2w2;   // log(g_{k+1}/g_k) = A - k B
    float gk = __expf(-dc * dc * i2w2);
    g[kc] = gk;
    float up = __expf(A - kc * B);
    float v = gk;
#pragma unroll
    for (int k = 0; k < DESC_RADIAL; ++k)
        if (k > kc) {
            v *= up;
            up *= F;
            g[k] = v;
        }
    float dn = __expf(-(A - (kc - 1) * B));          // g_{k-1} / g_k at k = kc
    v = gk;
#pragma unroll
    for (int k = DESC_RADIAL - 1; k >= 0; --k)
        if (k < kc) {
            v *= dn;
            dn *= F;
            g[k] = v;
        }
}

// one thread per slot; neighbours come from the column/cluster grid of the
// last pair-list build (the z extent of every cluster prunes a column)
__global__ void __launch_bounds__(128) k_descriptor(DevState st, const long long* __restrict__ fc,
                                                    float* __restrict__ feat) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots || st.orig[s] < 0) return;
    const int sysi = st.cluster_sys[s / CLUSTER];
    const SysDesc& sd = st.sys[sysi];
    const float4 xi = st.xyzq[s];
    const float L[3] = {sd.boxf[0], sd.boxf[1], sd.boxf[2]};
    const float iL[3] = {sd.inv_boxf[0], sd.inv_boxf[1], sd.inv_boxf[2]};
    float acc[4][DESC_RADIAL];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < DESC_RADIAL; ++k) acc[c][k] = 0.f;

    const float R = kDescReach;
    int cx0 = (int)floorf((xi.x - R) / sd.col_w[0]);
    int nx = (int)floorf((xi.x + R) / sd.col_w[0]) - cx0 + 1;
    if (nx >= sd.ncol_x) cx0 = 0, nx = sd.ncol_x;
    int cy0 = (int)floorf((xi.y - R) / sd.col_w[1]);
    int ny = (int)floorf((xi.y + R) / sd.col_w[1]) - cy0 + 1;
    if (ny >= sd.ncol_y) cy0 = 0, ny = sd.ncol_y;
    const float cut2 = DESC_CUT * DESC_CUT;
    constexpr float kPiF = 3.14159265358979f;
    for (int iy = 0; iy < ny; ++iy) {
        const int cy = wrap_col(cy0 + iy, sd.ncol_y);
        for (int ix = 0; ix < nx; ++ix) {
            const int cx = wrap_col(cx0 + ix, sd.ncol_x);
            const int col = sd.col_off + cx + sd.ncol_x * cy;
            const int j0 = st.col_cl_start[col], nj = st.col_ncl[col];
            for (int jc = j0; jc < j0 + nj; ++jc) {
                const float4 lo = st.bb_lo[jc], hi = st.bb_hi[jc];
                // z gap to the cluster's extent under the nearest periodic image
                const float zc = 0.5f * (lo.z + hi.z), ze = 0.5f * (hi.z - lo.z);
                float dzc = zc - xi.z;
                dzc -= L[2] * rintf(dzc * iL[2]);
                if (fabsf(dzc) - ze > R) continue;
                for (int k = 0; k < CLUSTER; ++k) {
                    const int sj = jc * CLUSTER + k;
                    if (sj == s || st.orig[sj] < 0) continue;
                    const float4 xj = st.xyzq[sj];
                    float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
                    dx -= L[0] * rintf(dx * iL[0]);
                    dy -= L[1] * rintf(dy * iL[1]);
                    dz -= L[2] * rintf(dz * iL[2]);
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 >= cut2 || r2 <= 0.f || xj.w == 0.f) continue;
                    const float r = sqrtf(r2);
                    const float w0 = xj.w * (1.f / kE) * 0.5f * (__cosf(kPiF * r / DESC_CUT) + 1.f);
                    const float ir = 1.f / r;
                    const float w[4] = {w0, w0 * dx * ir, w0 * dy * ir, w0 * dz * ir};
                    float g[DESC_RADIAL];
                    radial16(r, g);
#pragma unroll
                    for (int c = 0; c < 4; ++c)
#pragma unroll
                        for (int q = 0; q < DESC_RADIAL; ++q) acc[c][q] = fmaf(w[c], g[q], acc[c][q]);
                }
            }
        }
    }
    float* out = feat + (size_t)s * MLP_IN;
    const float inv = (float)(1.0 / FORCE_SCALE);
    out[0] = (float)fc[s] * inv;
    out[1] = (float)fc[st.n_slots + s] * inv;
    out[2] = (float)fc[2 * (size_t)st.n_slots + s] * inv;
    out[3] = xi.w;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < DESC_RADIAL; ++k) out[4 + DESC_RADIAL * c + k] = acc[c][k];
}

// normalised BF16 network input, rows padded from 68 to 80 columns with zeros
__global__ void k_mlp_input(int n_rows, const float* __restrict__ feat, const float* __restrict__ mean,
                            const float* __restrict__ inv_std, __nv_bfloat16* __restrict__ X) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)n_rows * MLP_KIN) return;
    const int r = (int)(i / MLP_KIN), c = (int)(i - (long long)r * MLP_KIN);
    float v = 0.f;
    if (c < MLP_IN) v = (feat[(size_t)r * MLP_IN + c] - mean[c]) * inv_std[c];
    X[i] = __float2bfloat16(v);
}

// forces += coarse force + scale * predicted residual (fixed point, atomics:
// the pair kernel adds into the same accumulators concurrently)
__global__ void k_mlp_apply(DevState st, const long long* __restrict__ fc, const float* __restrict__ Y,
                            float scale) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots || st.orig[s] < 0) return;
    const size_t n = st.n_slots;
    atomic_add_fixed(st.fx + s, fc[s] + to_fixed(Y[(size_t)s * 8 + 0] * scale, FORCE_SCALE));
    atomic_add_fixed(st.fy + s, fc[n + s] + to_fixed(Y[(size_t)s * 8 + 1] * scale, FORCE_SCALE));
    atomic_add_fixed(st.fz + s, fc[2 * n + s] + to_fixed(Y[(size_t)s * 8 + 2] * scale, FORCE_SCALE));
}

// training rows in original atom order: features and target = full - coarse
__global__ void k_collect(DevState st, const float* __restrict__ feat, const long long* __restrict__ fc,
                          const long long* __restrict__ ff, float* __restrict__ rows_feat,
                          float* __restrict__ rows_target) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots) return;
    const int a = st.orig[s];
    if (a < 0) return;
    const size_t n = st.n_slots;
    for (int c = 0; c < MLP_IN; ++c) rows_feat[(size_t)a * MLP_IN + c] = feat[(size_t)s * MLP_IN + c];
    const double inv = 1.0 / FORCE_SCALE;
    for (int d = 0; d < 3; ++d)
        rows_target[(size_t)a * 3 + d] = (float)((double)(ff[d * n + s] - fc[d * n + s]) * inv);
}

// one training batch: rows idx[i] of the collected frames, normalised
__global__ void k_gather_batch(const float* __restrict__ rows_feat, const float* __restrict__ rows_target,
                               const int* __restrict__ idx, int n, const float* __restrict__ mean,
                               const float* __restrict__ inv_std, float out_inv_scale,
                               __nv_bfloat16* __restrict__ X, float* __restrict__ T) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)n * MLP_KIN) return;
    const int r = (int)(i / MLP_KIN), c = (int)(i - (long long)r * MLP_KIN);
    const size_t src = (size_t)idx[r];
    float v = 0.f;
    if (c < MLP_IN) v = (rows_feat[src * MLP_IN + c] - mean[c]) * inv_std[c];
    X[i] = __float2bfloat16(v);
    if (c < 3) T[(size_t)r * 3 + c] = rows_target[src * 3 + c] * out_inv_scale;
}

// sums[0] += |fc + scale Y - ff|^2, sums[1] += |ff|^2, sums[2] += |fc - ff|^2
// (reciprocal forces only; the full-grid check of the running correction)
__global__ void k_pred_error(DevState st, const long long* __restrict__ fc, const float* __restrict__ Y,
                             float scale, const long long* __restrict__ ff, double* __restrict__ sums) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double e_l = 0.0, e_f = 0.0, e_c = 0.0;
    if (s < st.n_slots && st.orig[s] >= 0) {
        const size_t n = st.n_slots;
        const double inv = 1.0 / FORCE_SCALE;
        for (int d = 0; d < 3; ++d) {
            const double c = (double)fc[d * n + s] * inv, f = (double)ff[d * n + s] * inv;
            const double l = c + (double)Y[(size_t)s * 8 + d] * scale;
            e_l += (l - f) * (l - f);
            e_f += f * f;
            e_c += (c - f) * (c - f);
        }
    }
    e_l = warp_sum(e_l);
    e_f = warp_sum(e_f);
    e_c = warp_sum(e_c);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sums + 0, e_l);
        atomicAdd(sums + 1, e_f);
        atomicAdd(sums + 2, e_c);
    }
}

__global__ void k_add_forces(DevState st, const long long* __restrict__ src) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots || st.orig[s] < 0) return;
    const size_t n = st.n_slots;
    atomic_add_fixed(st.fx + s, src[s]);
    atomic_add_fixed(st.fy + s, src[n + s]);
    atomic_add_fixed(st.fz + s, src[2 * n + s]);
}

__global__ void k_rows_to_bf16(int n, const float* __restrict__ x, __nv_bfloat16* __restrict__ X) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)n * MLP_KIN) return;
    const int r = (int)(i / MLP_KIN), c = (int)(i - (long long)r * MLP_KIN);
    X[i] = __float2bfloat16(c < MLP_IN ? x[(size_t)r * MLP_IN + c] : 0.f);
}

int launch_descriptor(const DevState& st, const long long* fc, float* feat, cudaStream_t s) {
    k_descriptor<<<nblk(st.n_slots, 128), 128, 0, s>>>(st, fc, feat);
    return 1;
}
int launch_mlp_input(const DevState& st, const float* feat, const float* mean, const float* inv_std,
                     __nv_bfloat16* X, cudaStream_t s) {
    k_mlp_input<<<nblk((long long)st.n_slots * MLP_KIN, 256), 256, 0, s>>>(st.n_slots, feat, mean, inv_std, X);
    return 1;
}
int launch_mlp_apply(const DevState& st, const long long* fc, const float* Y, float out_scale, cudaStream_t s) {
    k_mlp_apply<<<nblk(st.n_slots, 256), 256, 0, s>>>(st, fc, Y, out_scale);
    return 1;
}
int launch_collect(const DevState& st, const float* feat, const long long* fc, const long long* ff,
                   float* rows_feat, float* rows_target, cudaStream_t s) {
    k_collect<<<nblk(st.n_slots, 256), 256, 0, s>>>(st, feat, fc, ff, rows_feat, rows_target);
    return 1;
}
int launch_gather_batch(const float* rows_feat, const float* rows_target, const int* idx, int n,
                        const float* mean, const float* inv_std, float out_inv_scale, __nv_bfloat16* X, float* T,
                        cudaStream_t s) {
    k_gather_batch<<<nblk((long long)n * MLP_KIN, 256), 256, 0, s>>>(rows_feat, rows_target, idx, n, mean, inv_std,
                                                                     out_inv_scale, X, T);
    return 1;
}
int launch_pred_error(const DevState& st, const long long* fc, const float* Y, float scale, const long long* ff,
                      double* sums, cudaStream_t s) {
    k_pred_error<<<nblk(st.n_slots, 256), 256, 0, s>>>(st, fc, Y, scale, ff, sums);
    return 1;
}
int launch_add_forces(const DevState& st, const long long* src, cudaStream_t s) {
    k_add_forces<<<nblk(st.n_slots, 256), 256, 0, s>>>(st, src);
    return 1;
}
int launch_rows_to_bf16(int n, const float* x, __nv_bfloat16* X, cudaStream_t s) {
    k_rows_to_bf16<<<nblk((long long)n * MLP_KIN, 256), 256, 0, s>>>(n, x, X);
    return 1;
}

}  // namespace lima
