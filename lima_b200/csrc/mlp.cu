// mlp.cu — the network of the learned coarse-grid PME correction.
//
// A small MLP (68 -> 128 -> 128 -> 128 -> 3, SiLU) maps each atom's coarse-grid
// reciprocal force (3), its charge (1) and a 64-value local descriptor to the
// residual between the full-grid and the coarse-grid reciprocal force.  The
// reference has no learned component.
//
// Layout: activations are row-major [rows][ld] BF16, one row per atom; weights
// are kept as FP32 masters W[K][N] (Adam state beside them) and as two BF16
// copies, W[K][N] and WT[N][K].  Every GEMM runs on the tensor cores through
// mma.sync m16n8k16 (BF16 inputs, FP32 accumulation); a CTA of 8 warps owns 128
// rows, a warp 16 rows and all N columns.  Weight and bias gradients are summed
// per chunk of MLP_CHUNK rows into partial buffers and reduced in chunk order,
// so training is deterministic.
#include <cuda_bf16.h>

#include <algorithm>

#include "engine.h"
#include "mlp.h"

namespace lima {

__device__ __forceinline__ void mma16816(float* c, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16* p) {
    return *reinterpret_cast<const uint32_t*>(p);
}
__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
// inference epilogues: silu(z) = z/2 (1 + tanh(z/2)) with the hardware tanh
// (PTX tanh.approx.f32, relative error ~2^-11, below the BF16 rounding of the result)
__device__ __forceinline__ float silu_fast(float z) {
    const float h = 0.5f * z;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
    return fmaf(h, t, h);
}
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.f / (1.f + __expf(-z));
    return s * (1.f + z * (1.f - s));
}

// ------------------------------------------------------------------ row GEMM
// C[rows][N] = A[rows][K] * B, with B given as BT[N][ldb] (row n holds B(:, n)).
// MODE 0: hidden layer forward   z = C + bias; Z <- z (if Zout), H <- silu(z)
// MODE 1: output layer forward   Y[row][0..7] <- C + bias (FP32)
// MODE 2: backward through SiLU  dZ <- C * silu'(Zprev[row][n])
template <int K, int N, int MODE>
__global__ void __launch_bounds__(256) k_gemm_rows(int rows, const __nv_bfloat16* __restrict__ A, int lda,
                                                   const __nv_bfloat16* __restrict__ BT, int ldb,
                                                   const float* __restrict__ bias, __nv_bfloat16* __restrict__ Zout,
                                                   __nv_bfloat16* __restrict__ Hout, int ldo,
                                                   float* __restrict__ Y, const __nv_bfloat16* __restrict__ Zprev) {
    constexpr int NT = N / 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = blockIdx.x * 128 + warp * 16;
    if (r0 >= rows) return;
    float acc[NT][4];
#pragma unroll
    for (int n = 0; n < NT; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
    const int ra = min(r0 + g, rows - 1), rb = min(r0 + g + 8, rows - 1);
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[4];
        a[0] = ld_pair(A + (size_t)ra * lda + k0 + 2 * t);
        a[1] = ld_pair(A + (size_t)rb * lda + k0 + 2 * t);
        a[2] = ld_pair(A + (size_t)ra * lda + k0 + 8 + 2 * t);
        a[3] = ld_pair(A + (size_t)rb * lda + k0 + 8 + 2 * t);
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            uint32_t b[2];
            const __nv_bfloat16* bp = BT + (size_t)(8 * n + g) * ldb + k0 + 2 * t;
            b[0] = ld_pair(bp);
            b[1] = ld_pair(bp + 8);
            mma16816(acc[n], a, b);
        }
    }
#pragma unroll
    for (int n = 0; n < NT; ++n) {
        const int c = 8 * n + 2 * t;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = r0 + g + 8 * h;
            if (r >= rows) continue;
            float v0 = acc[n][2 * h], v1 = acc[n][2 * h + 1];
            if (MODE == 0) {
                v0 += bias[c];
                v1 += bias[c + 1];
                if (Zout)
                    *reinterpret_cast<uint32_t*>(Zout + (size_t)r * ldo + c) =
                        pack2(__float2bfloat16(v0), __float2bfloat16(v1));
                *reinterpret_cast<uint32_t*>(Hout + (size_t)r * ldo + c) =
                    pack2(__float2bfloat16(silu(v0)), __float2bfloat16(silu(v1)));
            } else if (MODE == 1) {
                Y[(size_t)r * 8 + c] = v0 + bias[c];
                Y[(size_t)r * 8 + c + 1] = v1 + bias[c + 1];
            } else {
                const float z0 = __bfloat162float(Zprev[(size_t)r * ldo + c]);
                const float z1 = __bfloat162float(Zprev[(size_t)r * ldo + c + 1]);
                *reinterpret_cast<uint32_t*>(Hout + (size_t)r * ldo + c) =
                    pack2(__float2bfloat16(v0 * dsilu(z0)), __float2bfloat16(v1 * dsilu(z1)));
            }
        }
    }
}

// ------------------------------------------------------------- weight gradient
// part[chunk][K][N] = sum over the chunk's rows m of X[m][k] * dZ[m][n]
// (tensor cores: A = X^T, B = dZ; the row pairs (m, m+1) are gathered per lane)
template <int K, int N>
__global__ void __launch_bounds__(256) k_gemm_wgrad(int rows, const __nv_bfloat16* __restrict__ X, int ldx,
                                                    const __nv_bfloat16* __restrict__ dZ, int ldz,
                                                    float* __restrict__ part, int chunk) {
    constexpr int NT = N / 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int k0 = warp * 16;           // this warp's 16 rows of the K x N result
    if (k0 >= K) return;
    const int m_begin = blockIdx.x * chunk, m_end = min(rows, m_begin + chunk);
    float acc[NT][4];
#pragma unroll
    for (int n = 0; n < NT; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int m0 = m_begin; m0 < m_end; m0 += 16) {
        // A(r, c) = X[m0 + c][k0 + r]
        auto xa = [&](int r, int c) {
            const int m = m0 + c;
            return m < m_end ? X[(size_t)m * ldx + k0 + r] : zero;
        };
        uint32_t a[4];
        a[0] = pack2(xa(g, 2 * t), xa(g, 2 * t + 1));
        a[1] = pack2(xa(g + 8, 2 * t), xa(g + 8, 2 * t + 1));
        a[2] = pack2(xa(g, 2 * t + 8), xa(g, 2 * t + 9));
        a[3] = pack2(xa(g + 8, 2 * t + 8), xa(g + 8, 2 * t + 9));
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            // B(k, n) = dZ[m0 + k][n]
            auto zb = [&](int k, int col) {
                const int m = m0 + k;
                return m < m_end ? dZ[(size_t)m * ldz + col] : zero;
            };
            uint32_t b[2];
            b[0] = pack2(zb(2 * t, 8 * n + g), zb(2 * t + 1, 8 * n + g));
            b[1] = pack2(zb(2 * t + 8, 8 * n + g), zb(2 * t + 9, 8 * n + g));
            mma16816(acc[n], a, b);
        }
    }
    float* out = part + (size_t)blockIdx.x * K * N;
#pragma unroll
    for (int n = 0; n < NT; ++n) {
        const int c = 8 * n + 2 * t;
        out[(size_t)(k0 + g) * N + c] = acc[n][0];
        out[(size_t)(k0 + g) * N + c + 1] = acc[n][1];
        out[(size_t)(k0 + g + 8) * N + c] = acc[n][2];
        out[(size_t)(k0 + g + 8) * N + c + 1] = acc[n][3];
    }
}

// grad[i] = sum over chunks (fixed order) of part[chunk][i]
__global__ void k_reduce_parts(const float* __restrict__ part, int n_chunks, int n, float* __restrict__ grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.f;
    for (int c = 0; c < n_chunks; ++c) s += part[(size_t)c * n + i];
    grad[i] = s;
}

// bias-gradient partials: column sums of dZ over one chunk of rows per block
__global__ void k_colsum_part(int rows, const __nv_bfloat16* __restrict__ dZ, int ldz, int n, int chunk,
                              float* __restrict__ part) {
    const int c = threadIdx.x;
    if (c >= n) return;
    const int r0 = blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
    float s = 0.f;
    for (int r = r0; r < r1; ++r) s += __bfloat162float(dZ[(size_t)r * ldz + c]);
    part[(size_t)blockIdx.x * n + c] = s;
}

// ------------------------------------------------------------ loss, optimiser
// MSE over the 3 outputs; dZ4 = 2 (y - t) / (3 rows), padded to 16 columns
__global__ void k_mse(int rows, const float* __restrict__ Y, const float* __restrict__ T,
                      __nv_bfloat16* __restrict__ dZ4, double* __restrict__ loss) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (r < rows) {
        const float inv = 2.f / (3.f * (float)rows);
        for (int c = 0; c < 16; ++c) {
            float d = 0.f;
            if (c < 3) {
                const float e = Y[(size_t)r * 8 + c] - T[(size_t)r * 3 + c];
                l += (double)e * e;
                d = e * inv;
            }
            dZ4[(size_t)r * 16 + c] = __float2bfloat16(d);
        }
    }
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l);
}

__global__ void k_adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float c1, float c2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// BF16 copies of a master weight W[K][N]: W[K][ldw] and WT[N][ldt]
__global__ void k_to_bf16(const float* __restrict__ w, int K, int N, __nv_bfloat16* __restrict__ Wb, int ldw,
                          __nv_bfloat16* __restrict__ WTb, int ldt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= K * N) return;
    const int k = i / N, n = i - k * N;
    const __nv_bfloat16 b = __float2bfloat16(w[i]);
    if (Wb) Wb[(size_t)k * ldw + n] = b;
    if (WTb) WTb[(size_t)n * ldt + k] = b;
}

// ------------------------------------------------------- fused inference
// One persistent kernel for the whole network: the BF16 weights (transposed,
// rows padded by 8 elements so that ldmatrix rows fall on distinct banks) are
// loaded into shared memory once per CTA; each warp then streams 16-row tiles:
// normalise its 16 feature rows into shared memory, run the four layers with
// ldmatrix + mma.sync (activations stay in the warp's own 16 rows of shared
// memory), and write the 16 x 8 FP32 outputs.
constexpr int INF_WARPS = 16;
constexpr int LD1 = MLP_KIN + 8;     // 88
constexpr int LDH = MLP_HID + 8;     // 136
constexpr size_t INF_SMEM = sizeof(__nv_bfloat16) * ((size_t)128 * LD1 + 2 * (size_t)128 * LDH + 8 * (size_t)LDH +
                                                     (size_t)INF_WARPS * 16 * LDH) +
                            sizeof(float) * (3 * 128 + 8 + 2 * MLP_IN);

__device__ __forceinline__ void ldsm_x4(uint32_t* r, const __nv_bfloat16* p) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

// acc[16 x N] = A[16 x K] (rows of As, stride lda) * B, B given as BT[N][K] (stride ldb)
template <int K, int N>
__device__ __forceinline__ void warp_mma_tile(const __nv_bfloat16* As, int lda, const __nv_bfloat16* BT, int ldb,
                                              float (*acc)[4]) {
    const int lane = threadIdx.x & 31;
    const int mi = lane >> 3, rr = lane & 7;
#pragma unroll
    for (int n = 0; n < N / 8; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[4];
        ldsm_x4(a, As + (size_t)(rr + 8 * (mi & 1)) * lda + k0 + 8 * (mi >> 1));
        if (N >= 16) {
#pragma unroll
            for (int n = 0; n < N / 8; n += 2) {
                uint32_t b[4];
                ldsm_x4(b, BT + (size_t)(8 * (n + (mi >> 1)) + rr) * ldb + k0 + 8 * (mi & 1));
                mma16816(acc[n], a, b);
                mma16816(acc[n + 1], a, b + 2);
            }
        } else {
            // one n-tile: matrices (k0), (k0 + 8) of rows 0..7, loaded twice
            uint32_t b[4];
            ldsm_x4(b, BT + (size_t)rr * ldb + k0 + 8 * (mi & 1));
            mma16816(acc[0], a, b);
        }
    }
}

// bias + SiLU of a 16 x 128 accumulator tile into the warp's rows (BF16)
__device__ __forceinline__ void store_hidden(float (*acc)[4], const float* bias, __nv_bfloat16* H) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int n = 0; n < 16; ++n) {
        const int c = 8 * n + 2 * t;
        const float b0 = bias[c], b1 = bias[c + 1];
        *reinterpret_cast<uint32_t*>(H + (size_t)g * LDH + c) =
            pack2(__float2bfloat16(silu_fast(acc[n][0] + b0)), __float2bfloat16(silu_fast(acc[n][1] + b1)));
        *reinterpret_cast<uint32_t*>(H + (size_t)(g + 8) * LDH + c) =
            pack2(__float2bfloat16(silu_fast(acc[n][2] + b0)), __float2bfloat16(silu_fast(acc[n][3] + b1)));
    }
}

__global__ void __launch_bounds__(INF_WARPS * 32, 1)
    k_mlp_infer(int rows, const float* __restrict__ feat, const float* __restrict__ mean,
                const float* __restrict__ inv_std, const __nv_bfloat16* __restrict__ wt0,
                const __nv_bfloat16* __restrict__ wt1, const __nv_bfloat16* __restrict__ wt2,
                const __nv_bfloat16* __restrict__ wt3, const float* __restrict__ b0, const float* __restrict__ b1,
                const float* __restrict__ b2, const float* __restrict__ b3, float* __restrict__ Y) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __nv_bfloat16* W0 = reinterpret_cast<__nv_bfloat16*>(smem_raw);      // [128][LD1]
    __nv_bfloat16* W1 = W0 + 128 * LD1;                                   // [128][LDH]
    __nv_bfloat16* W2 = W1 + 128 * LDH;                                   // [128][LDH]
    __nv_bfloat16* W3 = W2 + 128 * LDH;                                   // [8][LDH]
    __nv_bfloat16* Hs = W3 + 8 * LDH;                                     // [warps][16][LDH]
    float* bs = reinterpret_cast<float*>(Hs + INF_WARPS * 16 * LDH);      // 3 x 128 + 8
    float* ms = bs + 3 * 128 + 8;                                         // mean, 1/std
    const int tid = threadIdx.x;
    for (int i = tid; i < 128 * MLP_KIN; i += blockDim.x) W0[(i / MLP_KIN) * LD1 + i % MLP_KIN] = wt0[i];
    for (int i = tid; i < 128 * 128; i += blockDim.x) {
        W1[(i >> 7) * LDH + (i & 127)] = wt1[i];
        W2[(i >> 7) * LDH + (i & 127)] = wt2[i];
    }
    for (int i = tid; i < 8 * 128; i += blockDim.x) W3[(i >> 7) * LDH + (i & 127)] = wt3[i];
    for (int i = tid; i < 128; i += blockDim.x) {
        bs[i] = b0[i];
        bs[128 + i] = b1[i];
        bs[256 + i] = b2[i];
    }
    if (tid < 8) bs[384 + tid] = b3[tid];
    for (int i = tid; i < MLP_IN; i += blockDim.x) {
        ms[i] = mean[i];
        ms[MLP_IN + i] = inv_std[i];
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    __nv_bfloat16* H = Hs + (size_t)warp * 16 * LDH;
    const int n_tiles = (rows + 15) / 16;
    float acc[16][4];
    for (int tile = blockIdx.x * INF_WARPS + warp; tile < n_tiles; tile += gridDim.x * INF_WARPS) {
        const int r0 = tile * 16;
        // 16 contiguous feature rows, normalised, into columns 0..79 (68..79 zero)
        for (int i = lane; i < 16 * MLP_KIN; i += 32) {
            const int r = i / MLP_KIN, c = i - r * MLP_KIN;
            float v = 0.f;
            if (c < MLP_IN && r0 + r < rows) v = (feat[(size_t)(r0 + r) * MLP_IN + c] - ms[c]) * ms[MLP_IN + c];
            H[r * LDH + c] = __float2bfloat16(v);
        }
        __syncwarp();
        warp_mma_tile<MLP_KIN, 128>(H, LDH, W0, LD1, acc);
        __syncwarp();
        store_hidden(acc, bs, H);
        __syncwarp();
        warp_mma_tile<128, 128>(H, LDH, W1, LDH, acc);
        __syncwarp();
        store_hidden(acc, bs + 128, H);
        __syncwarp();
        warp_mma_tile<128, 128>(H, LDH, W2, LDH, acc);
        __syncwarp();
        store_hidden(acc, bs + 256, H);
        __syncwarp();
        warp_mma_tile<128, 8>(H, LDH, W3, LDH, acc);
        const int g = lane >> 2, t = lane & 3;
        const int c = 2 * t;
        if (r0 + g < rows) {
            Y[(size_t)(r0 + g) * 8 + c] = acc[0][0] + bs[384 + c];
            Y[(size_t)(r0 + g) * 8 + c + 1] = acc[0][1] + bs[384 + c + 1];
        }
        if (r0 + g + 8 < rows) {
            Y[(size_t)(r0 + g + 8) * 8 + c] = acc[0][2] + bs[384 + c];
            Y[(size_t)(r0 + g + 8) * 8 + c + 1] = acc[0][3] + bs[384 + c + 1];
        }
        __syncwarp();
    }
}

// ------------------------------------------------ fused inference, tcgen05
// The same network on the 5th-generation tensor cores: one CTA (a warpgroup
// of 128 threads) per SM owns 128-row tiles.  All BF16 weights and the tile's
// activations sit in shared memory in the canonical K-major layout without
// swizzle (8-row x 16-byte core matrices: the two core matrices of one MMA's
// K = 16 are LBO = 128 B apart, consecutive 8-row groups SBO = K/8 x 128 B
// apart).  One thread issues tcgen05.mma (M = 128, N = 128 or 16, K = 16,
// BF16 x BF16 -> FP32) into 128 TMEM columns and commits to an mbarrier; after
// the wait, thread t of warp w reads row 32w + t of the accumulator with
// tcgen05.ld, adds the bias, applies SiLU and writes the next layer's input
// row back to shared memory.  Every wait on the mbarrier is bounded: on a
// timeout the kernel records an error, waits (bounded) once more for its MMAs
// and frees its TMEM before returning.
namespace tc {
constexpr int ROWS = 128;                              // rows per tile = TMEM lanes = one warpgroup
constexpr int GROUPS = 4;                              // warpgroups per CTA, each on its own tiles
constexpr int W0_OFF = 0;                              // N 128 x K 80
constexpr int W1_OFF = W0_OFF + 128 * 80 * 2;          // N 128 x K 128
constexpr int W2_OFF = W1_OFF + 128 * 128 * 2;
constexpr int W3_OFF = W2_OFF + 128 * 128 * 2;         // N 16 x K 128 (rows 8..15 zero)
constexpr int A_OFF = W3_OFF + 16 * 128 * 2;           // per group: 128 rows x K <= 128
constexpr int A_BYTES = ROWS * 128 * 2;
constexpr int BIAS_OFF = A_OFF + GROUPS * A_BYTES;     // 3 x 128 + 16 floats
constexpr int NORM_OFF = BIAS_OFF + (3 * 128 + 16) * 4;
constexpr int MBAR_OFF = NORM_OFF + 2 * MLP_IN * 4;    // one mbarrier per group, 8-byte aligned
constexpr int TADDR_OFF = MBAR_OFF + 8 * GROUPS;
constexpr int FLAG_OFF = TADDR_OFF + 4;                // one flag per group
constexpr int SMEM = FLAG_OFF + 4 * GROUPS;
constexpr int TMEM_COLS = 128 * GROUPS;
constexpr unsigned WAIT_LIMIT = 1u << 20;
static_assert(MBAR_OFF % 8 == 0, "mbarrier alignment");
static_assert(A_OFF % 16 == 0 && W3_OFF % 16 == 0, "16-byte aligned operands");

// byte offset of 16-byte chunk kc (elements 8kc..8kc+7) of row r, K columns
__device__ __forceinline__ int boff(int r, int kc, int K) { return ((r >> 3) * (K >> 3) + kc) * 128 + (r & 7) * 16; }

__device__ __forceinline__ uint64_t sdesc(unsigned saddr, int K) {
    const uint64_t lbo = 128 >> 4, sbo = (uint64_t)((K >> 3) * 128) >> 4;
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}
__host__ __device__ constexpr uint32_t idesc(int N) {
    // F32 accumulate, BF16 A and B, both K-major, N >> 3, M = 128 >> 4
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(id), "r"(accum), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void commit(unsigned mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ bool wait_parity(unsigned mbar, unsigned parity) {
    for (unsigned it = 0; it < WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// 16 columns of this thread's TMEM lane; the caller waits with ld_wait()
__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// barrier of one warpgroup (named barrier 1 + g, 128 threads)
__device__ __forceinline__ void group_sync(int g) { asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory"); }

// weights W^T[N][K] (row-major BF16) into the blocked layout; rows >= n_src are zero
__device__ void load_weights(unsigned char* dst, const __nv_bfloat16* src, int N, int K, int n_src) {
    const int kch = K >> 3;
    for (int c = threadIdx.x; c < N * kch; c += blockDim.x) {
        const int r = c / kch, kc = c - r * kch;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (r < n_src) v = *reinterpret_cast<const uint4*>(src + (size_t)r * K + 8 * kc);
        *reinterpret_cast<uint4*>(dst + boff(r, kc, K)) = v;
    }
}
}  // namespace tc

__global__ void __launch_bounds__(128 * tc::GROUPS, 1)
    k_mlp_infer_tc(int rows, const float* __restrict__ feat, const float* __restrict__ mean,
                   const float* __restrict__ inv_std, const __nv_bfloat16* __restrict__ wt0,
                   const __nv_bfloat16* __restrict__ wt1, const __nv_bfloat16* __restrict__ wt2,
                   const __nv_bfloat16* __restrict__ wt3, const float* __restrict__ b0, const float* __restrict__ b1,
                   const float* __restrict__ b2, const float* __restrict__ b3, float* __restrict__ Y,
                   int* __restrict__ err, int withhold) {
    using namespace tc;
    extern __shared__ __align__(128) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = tid / ROWS, gt = tid % ROWS;            // warpgroup, thread (= tile row) in it
    load_weights(sm + W0_OFF, wt0, 128, 80, 128);
    load_weights(sm + W1_OFF, wt1, 128, 128, 128);
    load_weights(sm + W2_OFF, wt2, 128, 128, 128);
    load_weights(sm + W3_OFF, wt3, 16, 128, 8);
    float* bias = reinterpret_cast<float*>(sm + BIAS_OFF);
    float* norm = reinterpret_cast<float*>(sm + NORM_OFF);
    for (int i = tid; i < 128; i += blockDim.x) {
        bias[i] = b0[i];
        bias[128 + i] = b1[i];
        bias[256 + i] = b2[i];
    }
    if (tid < 16) bias[384 + tid] = tid < 8 ? b3[tid] : 0.f;
    for (int i = tid; i < MLP_IN; i += blockDim.x) {
        norm[i] = mean[i];
        norm[MLP_IN + i] = inv_std[i];
    }
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(sm);
    const unsigned mbar = sbase + MBAR_OFF + 8 * g;
    volatile int* flag = reinterpret_cast<volatile int*>(sm + FLAG_OFF) + g;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + TADDR_OFF),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (gt == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1));
        *flag = 0;
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + TADDR_OFF) + 128u * g;   // this group's columns
    const uint32_t tmem_row = tmem + ((uint32_t)(32 * (warp & 3)) << 16);   // this warp's 32 lanes
    unsigned phase = 0;
    const int n_tiles = (rows + ROWS - 1) / ROWS;
    unsigned char* A = sm + A_OFF + g * A_BYTES;
    const unsigned a_addr = sbase + A_OFF + g * A_BYTES;
    const int wr0 = 32 * (warp & 3);                      // this warp's first row in the tile
    bool ok = true;
    for (int tile = GROUPS * blockIdx.x + g; tile < n_tiles && ok; tile += GROUPS * gridDim.x) {
        const int row = tile * ROWS + gt;
        // layer-1 input: the warp's 32 rows read as one contiguous block (coalesced),
        // normalised, K = 80 with 68..79 zero
        const size_t blk = (size_t)(tile * ROWS + wr0) * MLP_IN;
        const int nrow_w = min(32, rows - (tile * ROWS + wr0));
        // a row is 17 float4 (272 B, 16-byte aligned); four features -> one 8-byte store
        constexpr int Q = MLP_IN / 4;
#pragma unroll 4
        for (int i = lane; i < 32 * Q; i += 32) {
            const int r = i / Q, k = 4 * (i - r * Q);
            float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
            if (r < nrow_w) {
                f = *reinterpret_cast<const float4*>(feat + blk + (size_t)r * MLP_IN + k);
                f.x = (f.x - norm[k]) * norm[MLP_IN + k];
                f.y = (f.y - norm[k + 1]) * norm[MLP_IN + k + 1];
                f.z = (f.z - norm[k + 2]) * norm[MLP_IN + k + 2];
                f.w = (f.w - norm[k + 3]) * norm[MLP_IN + k + 3];
            }
            *reinterpret_cast<uint2*>(A + boff(wr0 + r, k >> 3, 80) + (k & 7) * 2) =
                make_uint2(pack2(__float2bfloat16(f.x), __float2bfloat16(f.y)),
                           pack2(__float2bfloat16(f.z), __float2bfloat16(f.w)));
        }
        // zero padding k = 68..79 of this thread's row (chunk 8 half, chunk 9)
        *reinterpret_cast<uint2*>(A + boff(gt, 8, 80) + 8) = make_uint2(0u, 0u);
        *reinterpret_cast<uint4*>(A + boff(gt, 9, 80)) = make_uint4(0u, 0u, 0u, 0u);
        fence_async_smem();
        group_sync(g);
#pragma unroll 1
        for (int l = 0; l < 4; ++l) {
            const int K = l == 0 ? 80 : 128, N = l == 3 ? 16 : 128;
            // withhold (a self-test of the bounded waits): the first layer's MMAs
            // and commit are not issued, so its wait runs out with nothing in flight
            if (gt == 0 && !(withhold && l == 0)) {
                const unsigned w_addr = sbase + (l == 0 ? W0_OFF : l == 1 ? W1_OFF : l == 2 ? W2_OFF : W3_OFF);
                fence_after();
                for (int ks = 0; ks < K / 16; ++ks)
                    tc::mma(tmem, sdesc(a_addr + ks * 256, K), sdesc(w_addr + ks * 256, K), idesc(N), ks > 0);
                commit(mbar);
            }
            // on a timeout `phase` stays the pending one, for the last wait below
            if (wait_parity(mbar, phase)) phase ^= 1u;
            else *flag = 1;
            group_sync(g);
            if (*flag) {
                ok = false;
                break;
            }
            fence_after();
            if (l < 3) {
                const float* bl = bias + 128 * l;
#pragma unroll 1
                for (int c4 = 0; c4 < 2; ++c4) {
                    uint32_t r[4][16];
#pragma unroll
                    for (int q = 0; q < 4; ++q) ld16(tmem_row + 64 * c4 + 16 * q, r[q]);
                    ld_wait();
#pragma unroll
                    for (int q = 0; q < 4; ++q)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int b = 64 * c4 + 16 * q + 8 * h;
                            float v[8];
#pragma unroll
                            for (int e = 0; e < 8; ++e) v[e] = silu_fast(__uint_as_float(r[q][8 * h + e]) + bl[b + e]);
                            uint4 u;
                            u.x = pack2(__float2bfloat16(v[0]), __float2bfloat16(v[1]));
                            u.y = pack2(__float2bfloat16(v[2]), __float2bfloat16(v[3]));
                            u.z = pack2(__float2bfloat16(v[4]), __float2bfloat16(v[5]));
                            u.w = pack2(__float2bfloat16(v[6]), __float2bfloat16(v[7]));
                            *reinterpret_cast<uint4*>(A + boff(gt, b >> 3, 128)) = u;
                        }
                }
            } else {
                uint32_t r[16];
                ld16(tmem_row, r);
                ld_wait();
                if (row < rows) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) Y[(size_t)row * 8 + j] = __uint_as_float(r[j]) + bias[384 + j];
                }
            }
            fence_before();
            fence_async_smem();
            group_sync(g);
        }
    }
    if (!ok) {
        if (gt == 0) atomicExch(err, 1);
        // let any MMA still in flight finish before the accumulator is freed
        wait_parity(mbar, phase);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(*reinterpret_cast<volatile uint32_t*>(sm + TADDR_OFF)), "r"(TMEM_COLS));
    }
}

// ---------------------------------------------------------- model host side
namespace {
inline unsigned blocks(long long n, int tb) { return (unsigned)((n + tb - 1) / tb); }
}  // namespace

void mlp_sync_bf16(MlpModel& m, cudaStream_t s) {
    for (int l = 0; l < 4; ++l) {
        const int K = MLP_K[l], N = MLP_N[l];
        // the last layer's W keeps 16 columns (8..15 zero) for the backward GEMM
        const int ldw = l == 3 ? 16 : N;
        k_to_bf16<<<blocks((long long)K * N, 256), 256, 0, s>>>(m.w[l], K, N, m.wb[l], ldw, m.wtb[l], K);
    }
}

int mlp_infer(const MlpModel& m, int rows, const float* feat, const float* mean, const float* inv_std, float* Y,
              cudaStream_t s) {
    static std::atomic<unsigned long long> attr_set{0ull};
    once_per_device(attr_set, [] {
        cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INF_SMEM);
    });
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (rows + 15) / 16;
    const int grid = std::max(1, std::min(sms, (tiles + INF_WARPS - 1) / INF_WARPS));
    k_mlp_infer<<<grid, INF_WARPS * 32, INF_SMEM, s>>>(rows, feat, mean, inv_std, m.wtb[0], m.wtb[1], m.wtb[2],
                                                       m.wtb[3], m.b[0], m.b[1], m.b[2], m.b[3], Y);
    return 1;
}

int mlp_infer_tc(const MlpModel& m, int rows, const float* feat, const float* mean, const float* inv_std, float* Y,
                 int* err, cudaStream_t s, int withhold) {
    static std::atomic<unsigned long long> attr_set{0ull};
    once_per_device(attr_set, [] {
        cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM);
    });
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (rows + tc::ROWS - 1) / tc::ROWS;
    const int grid = std::max(1, std::min(sms, (tiles + tc::GROUPS - 1) / tc::GROUPS));
    k_mlp_infer_tc<<<grid, 128 * tc::GROUPS, tc::SMEM, s>>>(rows, feat, mean, inv_std, m.wtb[0], m.wtb[1], m.wtb[2], m.wtb[3],
                                              m.b[0], m.b[1], m.b[2], m.b[3], Y, err, withhold);
    return 1;
}

int mlp_forward(const MlpModel& m, int rows, const __nv_bfloat16* X, MlpActs* acts, float* Y, cudaStream_t s) {
    const unsigned g = blocks(rows, 128);
    __nv_bfloat16* z[3] = {acts ? acts->z[0] : nullptr, acts ? acts->z[1] : nullptr, acts ? acts->z[2] : nullptr};
    __nv_bfloat16* h[3] = {acts ? acts->h[0] : m.tmp[0], acts ? acts->h[1] : m.tmp[1], acts ? acts->h[2] : m.tmp[0]};
    k_gemm_rows<MLP_KIN, 128, 0><<<g, 256, 0, s>>>(rows, X, MLP_KIN, m.wtb[0], MLP_KIN, m.b[0], z[0], h[0], 128,
                                                   nullptr, nullptr);
    k_gemm_rows<128, 128, 0><<<g, 256, 0, s>>>(rows, h[0], 128, m.wtb[1], 128, m.b[1], z[1], h[1], 128, nullptr,
                                               nullptr);
    k_gemm_rows<128, 128, 0><<<g, 256, 0, s>>>(rows, h[1], 128, m.wtb[2], 128, m.b[2], z[2], h[2], 128, nullptr,
                                               nullptr);
    k_gemm_rows<128, 8, 1><<<g, 256, 0, s>>>(rows, h[2], 128, m.wtb[3], 128, m.b[3], nullptr, nullptr, 8, Y,
                                             nullptr);
    return 4;
}

int mlp_train_step(MlpModel& m, int rows, const __nv_bfloat16* X, const float* T, MlpActs& a, float lr,
                   double* d_loss, cudaStream_t s) {
    int launches = mlp_forward(m, rows, X, &a, a.y, s);
    const unsigned g = blocks(rows, 128);
    k_mse<<<blocks(rows, 256), 256, 0, s>>>(rows, a.y, T, a.dz4, d_loss);
    const int chunk = MLP_CHUNK;
    const unsigned nch = blocks(rows, chunk);
    // layer 4: dW4 = H3^T dZ4 (first 8 of the 16 dZ4 columns), db4, dZ3
    k_gemm_wgrad<128, 8><<<nch, 256, 0, s>>>(rows, a.h[2], 128, a.dz4, 16, m.part, chunk);
    k_reduce_parts<<<blocks(128 * 8, 256), 256, 0, s>>>(m.part, nch, 128 * 8, m.gw[3]);
    k_colsum_part<<<nch, 128, 0, s>>>(rows, a.dz4, 16, 8, chunk, m.bpart);
    k_reduce_parts<<<1, 128, 0, s>>>(m.bpart, nch, 8, m.gb[3]);
    k_gemm_rows<16, 128, 2><<<g, 256, 0, s>>>(rows, a.dz4, 16, m.wb[3], 16, nullptr, nullptr, a.dz[2], 128, nullptr,
                                              a.z[2]);
    // layers 3 and 2
    for (int l = 2; l >= 1; --l) {
        k_gemm_wgrad<128, 128><<<nch, 256, 0, s>>>(rows, a.h[l - 1], 128, a.dz[l], 128, m.part, chunk);
        k_reduce_parts<<<blocks(128 * 128, 256), 256, 0, s>>>(m.part, nch, 128 * 128, m.gw[l]);
        k_colsum_part<<<nch, 128, 0, s>>>(rows, a.dz[l], 128, 128, chunk, m.bpart);
        k_reduce_parts<<<1, 128, 0, s>>>(m.bpart, nch, 128, m.gb[l]);
        k_gemm_rows<128, 128, 2><<<g, 256, 0, s>>>(rows, a.dz[l], 128, m.wb[l], 128, nullptr, nullptr, a.dz[l - 1],
                                                   128, nullptr, a.z[l - 1]);
    }
    // layer 1: dW1 = X^T dZ1
    k_gemm_wgrad<MLP_KIN, 128><<<nch, 256, 0, s>>>(rows, X, MLP_KIN, a.dz[0], 128, m.part, chunk);
    k_reduce_parts<<<blocks(MLP_KIN * 128, 256), 256, 0, s>>>(m.part, nch, MLP_KIN * 128, m.gw[0]);
    k_colsum_part<<<nch, 128, 0, s>>>(rows, a.dz[0], 128, 128, chunk, m.bpart);
    k_reduce_parts<<<1, 128, 0, s>>>(m.bpart, nch, 128, m.gb[0]);
    launches += 21;
    if (lr > 0.f) {
        ++m.adam_step;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f / (1.f - powf(b1, (float)m.adam_step));
        const float c2 = 1.f / (1.f - powf(b2, (float)m.adam_step));
        for (int l = 0; l < 4; ++l) {
            const int nw = MLP_K[l] * MLP_N[l];
            k_adam<<<blocks(nw, 256), 256, 0, s>>>(nw, m.w[l], m.gw[l], m.mw[l], m.vw[l], lr, b1, b2, c1, c2, 1e-8f);
            k_adam<<<1, 128, 0, s>>>(MLP_N[l], m.b[l], m.gb[l], m.mb[l], m.vb[l], lr, b1, b2, c1, c2, 1e-8f);
        }
        mlp_sync_bf16(m, s);
        launches += 12;
    }
    return launches;
}

}  // namespace lima
