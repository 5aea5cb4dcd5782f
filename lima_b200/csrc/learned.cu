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
    const float gk = __expf(-dc * dc * i2w2);
    // every index below is static (the loops unroll), so g stays in registers
    float up = __expf(A - kc * B);
    float v = gk;
#pragma unroll
    for (int k = 0; k < DESC_RADIAL; ++k) {
        if (k == kc) g[k] = gk;
        if (k > kc) {
            v *= up;
            up *= F;
            g[k] = v;
        }
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

// One warp per i-cluster.  Lane (ii = lane & 7, jq = lane >> 3) owns i-atom ii
// and the j-atoms jq and jq + 4 of every candidate j-cluster; candidates come
// from the column grid of the last pair-list build in units of up to 32
// clusters of one column (one per lane), tested against the i-cluster's
// extent, staged in shared memory with one round of loads and then visited in
// order by the whole warp (so the warp never diverges on the walk).  The next
// unit's extents are requested before the current unit is evaluated.
constexpr int DS_WARPS = 4;

__global__ void __launch_bounds__(DS_WARPS * 32, 3) k_descriptor(DevState st, const long long* __restrict__ fc,
                                                                 float* __restrict__ feat) {
    __shared__ float4 stage_x[DS_WARPS][32][CLUSTER];
    const int ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (ci >= st.n_clusters) return;
    const int sysi = st.cluster_sys[ci];
    const SysDesc& sd = st.sys[sysi];
    if (ci - sd.cluster_cap_off >= st.sys_nclusters[sysi]) return;
    const float4 ilo = st.bb_lo[ci], ihi = st.bb_hi[ci];
    if (ilo.w == 0.f) return;   // empty cluster
    const int ii = lane & 7, jq = lane >> 3;
    const int si = ci * CLUSTER + ii;
    const bool ivalid = st.orig[si] >= 0;
    const float4 xi = st.xyzq[si];
    const float L[3] = {sd.boxf[0], sd.boxf[1], sd.boxf[2]};
    const float iL[3] = {sd.inv_boxf[0], sd.inv_boxf[1], sd.inv_boxf[2]};
    const float ic[3] = {0.5f * (ilo.x + ihi.x), 0.5f * (ilo.y + ihi.y), 0.5f * (ilo.z + ihi.z)};
    const float ie[3] = {0.5f * (ihi.x - ilo.x), 0.5f * (ihi.y - ilo.y), 0.5f * (ihi.z - ilo.z)};
    float acc[4][DESC_RADIAL];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < DESC_RADIAL; ++k) acc[c][k] = 0.f;

    const float R = kDescReach, R2 = R * R;
    int cx0 = (int)floorf((ilo.x - R) / sd.col_w[0]);
    int nx = (int)floorf((ihi.x + R) / sd.col_w[0]) - cx0 + 1;
    if (nx >= sd.ncol_x) cx0 = 0, nx = sd.ncol_x;
    int cy0 = (int)floorf((ilo.y - R) / sd.col_w[1]);
    int ny = (int)floorf((ihi.y + R) / sd.col_w[1]) - cy0 + 1;
    if (ny >= sd.ncol_y) cy0 = 0, ny = sd.ncol_y;
    const int ncw = nx * ny;
    auto header = [&](int k, int& j0, int& nj) {
        const int iy = k / nx, ix = k - iy * nx;
        const int col = sd.col_off + wrap_col(cx0 + ix, sd.ncol_x) + sd.ncol_x * wrap_col(cy0 + iy, sd.ncol_y);
        j0 = st.col_cl_start[col];
        nj = st.col_ncl[col];
    };
    const float cut2 = DESC_CUT * DESC_CUT;
    constexpr float kPiF = 3.14159265358979f;
    int k = 0, b = 0, j0 = 0, nj = 0;
    while (k < ncw) {
        header(k, j0, nj);
        if (nj > 0) break;
        ++k;
    }
    float4 jlo = make_float4(0.f, 0.f, 0.f, 0.f), jhi = jlo;
    if (k < ncw && lane < nj) {
        jlo = st.bb_lo[j0 + lane];
        jhi = st.bb_hi[j0 + lane];
    }
    while (k < ncw) {
        const int jc_lane = j0 + b + lane;
        bool pass = false;
        if (b + lane < nj && jlo.w != 0.f) {
            // gap between the two extents under the nearest periodic image
            const float jcx = 0.5f * (jlo.x + jhi.x) - ic[0], jcy = 0.5f * (jlo.y + jhi.y) - ic[1],
                        jcz = 0.5f * (jlo.z + jhi.z) - ic[2];
            const float d0 = fabsf(jcx - L[0] * rintf(jcx * iL[0])) - ie[0] - 0.5f * (jhi.x - jlo.x);
            const float d1 = fabsf(jcy - L[1] * rintf(jcy * iL[1])) - ie[1] - 0.5f * (jhi.y - jlo.y);
            const float d2 = fabsf(jcz - L[2] * rintf(jcz * iL[2])) - ie[2] - 0.5f * (jhi.z - jlo.z);
            const float a0 = fmaxf(d0, 0.f), a1 = fmaxf(d1, 0.f), a2 = fmaxf(d2, 0.f);
            pass = a0 * a0 + a1 * a1 + a2 * a2 < R2;
        }
        unsigned cand = __ballot_sync(0xffffffffu, pass);
        if (pass) {
#pragma unroll
            for (int a = 0; a < CLUSTER; ++a) stage_x[wib][lane][a] = st.xyzq[jc_lane * CLUSTER + a];
        }
        b += 32;
        if (b >= nj) {
            b = 0;
            ++k;
            while (k < ncw) {
                header(k, j0, nj);
                if (nj > 0) break;
                ++k;
            }
        }
        if (k < ncw && b + lane < nj) {
            jlo = st.bb_lo[j0 + b + lane];
            jhi = st.bb_hi[j0 + b + lane];
        }
        __syncwarp();
        while (cand) {
            const int src = __ffs(cand) - 1;
            cand &= cand - 1u;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float4 xj = stage_x[wib][src][jq + 4 * h];
                float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
                dx -= L[0] * rintf(dx * iL[0]);
                dy -= L[1] * rintf(dy * iL[1]);
                dz -= L[2] * rintf(dz * iL[2]);
                const float r2 = dx * dx + dy * dy + dz * dz;
                // padding slots carry q = 0, so the charge test drops them too
                const bool hit = ivalid && r2 < cut2 && r2 > 0.f && xj.w != 0.f;
                if (!__any_sync(0xffffffffu, hit)) continue;
                if (hit) {
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
        __syncwarp();
    }
    // sum the four lanes of each i-atom (fixed order), then lane jq writes channel jq
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < DESC_RADIAL; ++k) {
            float v = acc[c][k];
            v += __shfl_xor_sync(0xffffffffu, v, 8);
            v += __shfl_xor_sync(0xffffffffu, v, 16);
            acc[c][k] = v;
        }
    if (!ivalid) return;
    float* out = feat + (size_t)si * MLP_IN;
#pragma unroll
    for (int c = 0; c < 4; ++c)
        if (c == jq)
#pragma unroll
            for (int k = 0; k < DESC_RADIAL; ++k) out[4 + DESC_RADIAL * c + k] = acc[c][k];
    if (jq == 0) {
        const float inv = (float)(1.0 / FORCE_SCALE);
        out[0] = (float)fc[si] * inv;
        out[1] = (float)fc[st.n_slots + si] * inv;
        out[2] = (float)fc[2 * (size_t)st.n_slots + si] * inv;
        out[3] = xi.w;
    }
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
    k_descriptor<<<nblk((long long)st.n_clusters * 32, DS_WARPS * 32), DS_WARPS * 32, 0, s>>>(st, fc, feat);
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
