// pme.cu — smooth PME reciprocal space, order 4.
//
// Replaces PME::Controller::CalcCharges (code/LIMA_ENGINE/src/PME.cuh:574-608):
//   DistributeCompoundchargesToBlocksKernel + ChargeblockDistributeToGrid (:172-333)
//       -> k_spread: every atom adds q*w to its 4^3 grid nodes as int32 fixed
//          point (as the reference does, in 1 nm^3 shared tiles: an order-free,
//          deterministic sum; here straight into the L2-resident grid)
//   cufftExecR2C / ApplyGreensFunctionKernel / cufftExecC2R / Normalize (:585-599)
//       -> five shared-memory passes of a hand-written mixed-radix (2,3,4,5)
//          Stockham FFT: x (real->half complex), y, z (forward, x theta(k),
//          inverse, fused), y, x (half complex->real).  theta already holds
//          the 1/N normalisation.
//   InterpolateForcesAndPotentialKernel (:335-430)
//       -> k_gather: analytic B-spline derivative (accurate mode) or the
//          reference's central difference of the gridded potential.
// B-spline weights sit on nodes floor(u)-1..floor(u)+2 exactly as in
// ChargeblockDistributeToGrid (PME.cuh:249-300) and LAL::CalcBspline
// (DeviceAlgorithmsPrivate.cuh:7-30).
#include <algorithm>
#include <mutex>

#include "engine.h"
#include "lima_b200.h"

namespace lima {

constexpr int FFT_MAXN = 256;
constexpr int FFT_TX = PME_FFT_TX;          // columns per y/z tile
constexpr int FFT_XLINES = PME_FFT_XLINES;  // lines per x-pass CTA
constexpr int FFT_YZ_THREADS = 256;         // threads per y/z tile

struct FftPlanDev {
    int n;
    int nrad;
    int rad[12];
    int tw_off;  // offset of this length's twiddle table in DevState::pme_tw (-1: compute)
};

struct PmeSysDev {
    FftPlanDev px, py, pz;
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by sigma*i
__device__ __forceinline__ float2 mul_si(float2 a, float sigma) { return make_float2(-sigma * a.y, sigma * a.x); }

// R-point DFT in registers; sigma = -1 forward, +1 inverse
template <int R>
__device__ __forceinline__ void small_dft(float2* v, float sigma) {
    if (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 3) {
        const float s3 = 0.86602540378443865f;
        const float2 a = cadd(v[1], v[2]), b = csub(v[1], v[2]);
        const float2 m = csub(v[0], cscale(a, 0.5f));
        const float2 t = mul_si(b, sigma * s3);
        v[0] = cadd(v[0], a);
        v[1] = cadd(m, t);
        v[2] = csub(m, t);
    } else if (R == 4) {
        const float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        const float2 t2 = cadd(v[1], v[3]), t3 = mul_si(csub(v[1], v[3]), sigma);
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    } else if (R == 5) {
        const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
        const float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;
        const float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
        const float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
        const float2 x0 = v[0];
        const float2 m1 = cadd(x0, cadd(cscale(a1, c1), cscale(a2, c2)));
        const float2 m2 = cadd(x0, cadd(cscale(a1, c2), cscale(a2, c1)));
        const float2 n1 = mul_si(cadd(cscale(b1, s1), cscale(b2, s2)), sigma);
        const float2 n2 = mul_si(csub(cscale(b1, s2), cscale(b2, s1)), sigma);
        v[0] = cadd(x0, cadd(a1, a2));
        v[1] = cadd(m1, n1);
        v[4] = csub(m1, n1);
        v[2] = cadd(m2, n2);
        v[3] = csub(m2, n2);
    } else if (R == 8) {
        // two 4-point transforms (even and odd samples) joined by the eighth roots
        // of unity w^k = e^{sigma 2 pi i k / 8}: 1, (1 + sigma i)/sqrt 2, sigma i, (-1 + sigma i)/sqrt 2
        float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        small_dft<4>(e, sigma);
        small_dft<4>(o, sigma);
        const float r = 0.70710678118654752f;
        const float2 o1 = make_float2(r * (o[1].x - sigma * o[1].y), r * (o[1].y + sigma * o[1].x));
        const float2 o2 = mul_si(o[2], sigma);
        const float2 o3 = make_float2(r * (-o[3].x - sigma * o[3].y), r * (-o[3].y + sigma * o[3].x));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
}

// floor(a / b) for 0 <= a < 2^20, b >= 1, with inv_b = 1.0f / b: (a + 1/2) / b sits at
// least 1/(2b) from an integer and the two roundings of the product err by less
// than 2^-23 (a + 1/2) / b < 1/(8b), so the truncation is exact
__device__ __forceinline__ int div_small(int a, float inv_b) { return (int)(((float)a + 0.5f) * inv_b); }

template <int R>
__device__ __forceinline__ void stockham_stage(const float2* src, float2* dst, int nlines, int stride,
                                               int N, int Ns, const float2* tw, float sigma) {
    const int nb = N / R;
    const int total = nlines * nb;
    const int tscale = N / (Ns * R);
    const float inv_nb = 1.f / (float)nb, inv_ns = 1.f / (float)Ns;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int line = div_small(idx, inv_nb);
        const int j = idx - line * nb;
        const float2* in = src + line * stride;
        float2* out = dst + line * stride;
        const int jm = j - Ns * div_small(j, inv_ns);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[j + r * nb];
        // jm < Ns, so tstep * r <= (N/R)(R-1) < N: the twiddle index needs no wrap
        const int tstep = jm * tscale;
#pragma unroll
        for (int r = 1; r < R; ++r) {
            float2 w = tw[tstep * r];
            w.y *= -sigma;  // table holds e^{-2 pi i k/N}; conjugate for the inverse
            v[r] = cmul(v[r], w);
        }
        small_dft<R>(v, sigma);
        const int base = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) out[base + r * Ns] = v[r];
    }
}

// FFT of nlines lines (length pl.n, line stride `stride`) held in smem buffer a;
// b is scratch of the same size.  Returns the buffer holding the result.
__device__ float2* fft_lines(float2* a, float2* b, int nlines, int stride, const FftPlanDev& pl,
                             const float2* tw, float sigma) {
    float2* src = a;
    float2* dst = b;
    int Ns = 1;
    for (int s = 0; s < pl.nrad; ++s) {
        const int R = pl.rad[s];
        switch (R) {
            case 2: stockham_stage<2>(src, dst, nlines, stride, pl.n, Ns, tw, sigma); break;
            case 3: stockham_stage<3>(src, dst, nlines, stride, pl.n, Ns, tw, sigma); break;
            case 4: stockham_stage<4>(src, dst, nlines, stride, pl.n, Ns, tw, sigma); break;
            case 8: stockham_stage<8>(src, dst, nlines, stride, pl.n, Ns, tw, sigma); break;
            default: stockham_stage<5>(src, dst, nlines, stride, pl.n, Ns, tw, sigma); break;
        }
        __syncthreads();
        float2* t = src;
        src = dst;
        dst = t;
        Ns *= R;
    }
    return src;
}

__device__ void make_twiddles(float2* tw, int n) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double s, c;
        sincospi(2.0 * k / n, &s, &c);
        tw[k] = make_float2((float)c, (float)-s);
    }
}

// e^{-2 pi i k/n} from the table built at set-up (FP64 -> float), else computed
__device__ __forceinline__ void load_twiddles(float2* tw, const FftPlanDev& pl, const float2* table) {
    if (pl.tw_off >= 0 && table) {
        for (int k = threadIdx.x; k < pl.n; k += blockDim.x) tw[k] = table[pl.tw_off + k];
    } else {
        make_twiddles(tw, pl.n);
    }
}

// ------------------------------------------------------------------ spread
__device__ __forceinline__ void bspline4(float f, float* w) {
    const float g = 1.f - f;
    w[0] = g * g * g * (1.f / 6.f);
    w[1] = (4.f - 6.f * f * f + 3.f * f * f * f) * (1.f / 6.f);
    w[2] = (1.f + 3.f * f + 3.f * f * f - 3.f * f * f * f) * (1.f / 6.f);
    w[3] = f * f * f * (1.f / 6.f);
}
__device__ __forceinline__ void bspline4_d(float f, float* dw) {
    const float g = 1.f - f;
    dw[0] = -0.5f * g * g;
    dw[1] = -2.f * f + 1.5f * f * f;
    dw[2] = 0.5f + f - 1.5f * f * f;
    dw[3] = 0.5f * f * f;
}

__device__ __forceinline__ int wrapk(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}
// element c of a 4-array for a c known only at run time, without local memory
__device__ __forceinline__ float pick4(const float (&w)[4], int c) {
    return c == 0 ? w[0] : (c == 1 ? w[1] : (c == 2 ? w[2] : w[3]));
}
// i mod n for i in [-n, 2n): a node index at most one period outside the grid
__device__ __forceinline__ int wrap1(int i, int n) {
    return i < 0 ? i + n : (i >= n ? i - n : i);
}

// grid coordinate in [0,K): integer base and fraction.  Positions lie within a
// box length of the box (wrapped at every list build, drifting a little
// between builds), so one add or subtract of K brings u into range; anything
// else (far away or non-finite) takes the general reduction.
__device__ __forceinline__ void grid_coord(float x, float inv_h, int K, int& base, float& frac) {
    float u = x * inv_h;
    const float Kf = (float)K;
    if (u < 0.f) u += Kf;
    else if (u >= Kf) u -= Kf;
    if (!(u >= 0.f && u < Kf)) u -= Kf * floorf(u / Kf);
    float fl = floorf(u);
    base = (int)fl;
    frac = u - fl;
    if (base >= K) base -= K;
    if (!(base >= 0 && base < K)) {  // non-finite position: keep the index in range
        base = 0;
        frac = 0.f;
    }
}

// four threads per atom, one per z-plane of the 4x4x4 stencil
__global__ void k_spread(DevState st) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = t >> 2, c = t & 3;
    if (s >= st.n_slots) return;
    const float4 p = st.xyzq[s];
    if (p.w == 0.f || st.orig[s] < 0) return;
    const SysDesc& sd = st.sys[st.cluster_sys[s / CLUSTER]];
    if (sd.pme_n[0] == 0) return;
    const int K0 = sd.pme_n[0], K1 = sd.pme_n[1], K2 = sd.pme_n[2];
    int b0, b1, b2;
    float f0, f1, f2;
    grid_coord(p.x, sd.pme_inv_h[0], K0, b0, f0);
    grid_coord(p.y, sd.pme_inv_h[1], K1, b1, f1);
    grid_coord(p.z, sd.pme_inv_h[2], K2, b2, f2);
    float wx[4], wy[4], wz[4];
    bspline4(f0, wx);
    bspline4(f1, wy);
    bspline4(f2, wz);
    int* g = st.pme_grid_fx + sd.pme_off;
    int ix[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) ix[a] = wrap1(b0 - 1 + a, K0);
    const int z = wrap1(b2 - 1 + c, K2);
    const float qz = p.w * pick4(wz, c);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int y = wrap1(b1 - 1 + b, K1);
        const float qyz = qz * wy[b];
        int* row = g + (size_t)K0 * (y + (size_t)K1 * z);
#pragma unroll
        for (int a = 0; a < 4; ++a) atomicAdd(row + ix[a], __float2int_rn(qyz * wx[a] * (float)GRID32_SCALE));
    }
}

// Spreading by column blocks.  One CTA per item (system, block of
// PME_SPREAD_COLS^2 columns of the pair-search grid, chunk of z nodes — the whole
// z range unless the box would not fit): every charged atom of the block's
// columns adds its 4^3 weighted charges, owned by the item's z chunk, into a
// shared-memory box of nodes, and the box goes to the grid once, x-contiguous,
// empty nodes skipped.  On a 0.1 nm grid with 0.43 nm columns a column's 12,000
// weights land on about 5,000 nodes, so the grid sees 40 % of the atomics of one
// per weight, coalesced.  A weight outside the box (an atom that drifted from its
// column since the list build, or a grid too fine for the box) is added to the
// grid directly.  Every weight is the same int32 as in k_spread, so the grid
// holds the same integers.
int pme_spread_box_side(double col_w, double inv_h) {
    // stencil start floor(u) - 1 with u in [u_lo, u_hi): nodes floor(u_lo) - 1 ..
    // floor(u_hi) + 2, at most ceil(u_hi - u_lo) + 4 of them; one more for rounding
    return (int)std::ceil(PME_SPREAD_COLS * col_w * inv_h) + 5;
}

__global__ void __launch_bounds__(256) k_spread_tiles(DevState st, const int4* items, const int4* geo) {
    extern __shared__ __align__(16) int sbox[];
    const int4 it = items[blockIdx.x];
    const SysDesc& sd = st.sys[it.x];
    const int4 gm = geo[it.x];
    const int NX = gm.x, NY = gm.y, ZC = gm.z;
    const int K0 = sd.pme_n[0], K1 = sd.pme_n[1], K2 = sd.pme_n[2];
    const int z0 = it.w, nz = min(ZC, K2 - z0);
    const int nbox = NX * NY * ZC;
    // clear the box, 16 bytes per store (dynamic shared memory starts 16-byte aligned)
    for (int i = threadIdx.x; i < nbox / 4; i += blockDim.x) reinterpret_cast<int4*>(sbox)[i] = make_int4(0, 0, 0, 0);
    for (int i = (nbox & ~3) + threadIdx.x; i < nbox; i += blockDim.x) sbox[i] = 0;
    // box origin: the stencil start of an atom on the block's lower edge
    const int ox = (int)floorf((float)it.y * sd.col_w[0] * sd.pme_inv_h[0]) - 1;
    const int oy = (int)floorf((float)it.z * sd.col_w[1] * sd.pme_inv_h[1]) - 1;
    __syncthreads();
    int* g = st.pme_grid_fx + sd.pme_off;
    const int cx1 = min(it.y + PME_SPREAD_COLS, sd.ncol_x), cy1 = min(it.z + PME_SPREAD_COLS, sd.ncol_y);
    for (int cy = it.z; cy < cy1; ++cy) {
        for (int cx = it.y; cx < cx1; ++cx) {
            const int col = sd.col_off + cx + sd.ncol_x * cy;
            const int s0 = st.col_cl_start[col] * CLUSTER;
            const int ns = st.col_ncl[col] * CLUSTER;
            // four threads per atom, one per z node of its stencil
            for (int t = threadIdx.x; t < 4 * ns; t += blockDim.x) {
                const int s = s0 + (t >> 2), c = t & 3;
                const float4 p = st.xyzq[s];
                if (p.w == 0.f || st.orig[s] < 0) continue;
                int b0, b1, b2;
                float f0, f1, f2;
                grid_coord(p.z, sd.pme_inv_h[2], K2, b2, f2);
                const int z = wrap1(b2 - 1 + c, K2);
                const int lz = z - z0;
                if (lz < 0 || lz >= nz) continue;   // another item's chunk
                grid_coord(p.x, sd.pme_inv_h[0], K0, b0, f0);
                grid_coord(p.y, sd.pme_inv_h[1], K1, b1, f1);
                float wx[4], wy[4], wz[4];
                bspline4(f0, wx);
                bspline4(f1, wy);
                bspline4(f2, wz);
                // box-relative stencil start; b0 is wrapped into [0, K0), so take
                // the periodic image nearest the box
                int lx = b0 - 1 - ox, ly = b1 - 1 - oy;
                if (lx < -K0 / 2) lx += K0;
                else if (lx > NX + K0 / 2) lx -= K0;
                if (ly < -K1 / 2) ly += K1;
                else if (ly > NY + K1 / 2) ly -= K1;
                // the fixed-point scale is a power of two, so taking it into the
                // charge first gives every product that can round to a non-zero
                // integer exactly as q w_z w_y w_x scaled last (k_spread's order)
                const float qz = p.w * pick4(wz, c) * (float)GRID32_SCALE;
                if (lx >= 0 && lx + 3 < NX && ly >= 0 && ly + 3 < NY) {
                    int* node = sbox + lx + NX * (ly + NY * lz);
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const float qyz = qz * wy[b];
#pragma unroll
                        for (int a = 0; a < 4; ++a) atomicAdd(node + a + NX * b, __float2int_rn(qyz * wx[a]));
                    }
                } else {
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const float qyz = qz * wy[b];
                        int* row = g + (size_t)K0 * (wrap1(b1 - 1 + b, K1) + (size_t)K1 * z);
#pragma unroll
                        for (int a = 0; a < 4; ++a) atomicAdd(row + wrap1(b0 - 1 + a, K0), __float2int_rn(qyz * wx[a]));
                    }
                }
            }
        }
    }
    __syncthreads();
    // one thread per (x, y) column of the box and group of eight z nodes:
    // consecutive threads add to consecutive x nodes of the grid
    const int nxy = NX * NY, ngz = (nz + 7) >> 3;
    const size_t zs = (size_t)K0 * K1;
    if (nxy <= (int)blockDim.x) {
        // each thread keeps one column and strides over its z groups (no division per group)
        const int tpc = blockDim.x / nxy;
        const int c = threadIdx.x % nxy, g0 = threadIdx.x / nxy;
        if (g0 < tpc) {
            const int ix = c % NX, iy = c / NX;
            const int x = NX <= K0 ? wrap1(ox + ix, K0) : wrapk(ox + ix, K0);
            const int y = NY <= K1 ? wrap1(oy + iy, K1) : wrapk(oy + iy, K1);
            int* gcol = g + x + (size_t)K0 * y + zs * z0;
            for (int gz = g0; gz < ngz; gz += tpc) {
                const int iz0 = gz << 3, m = min(8, nz - iz0);
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (u < m) {
                        const int v = sbox[c + nxy * (iz0 + u)];
                        if (v != 0) atomicAdd(gcol + zs * (iz0 + u), v);
                    }
                }
            }
        }
        return;
    }
    for (int i = threadIdx.x; i < nxy * ngz; i += blockDim.x) {
        const int c = i % nxy, iz0 = (i / nxy) << 3;
        const int ix = c % NX, iy = c / NX;
        // ox, oy >= -1 and below K - 1: one period unless the box is wider than the grid
        const int x = NX <= K0 ? wrap1(ox + ix, K0) : wrapk(ox + ix, K0);
        const int y = NY <= K1 ? wrap1(oy + iy, K1) : wrapk(oy + iy, K1);
        int* gcol = g + x + (size_t)K0 * y + zs * (z0 + iz0);
        const int m = min(8, nz - iz0);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (u < m) {
                const int v = sbox[c + nxy * (iz0 + u)];
                if (v != 0) atomicAdd(gcol + zs * u, v);
            }
        }
    }
}

// ------------------------------------------------------------- FFT passes
// Copies `total` elements with the whole block, four independent loads per
// thread in flight before their stores (the passes are bound by load latency):
// load(i) returns element i, store(i, v) places it.
template <typename T, typename Load, typename Store>
__device__ __forceinline__ void block_copy4(int total, Load load, Store store) {
    for (int i0 = threadIdx.x; i0 < total; i0 += 4 * blockDim.x) {
        T v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < total) v[u] = load(i);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < total) store(i, v[u]);
        }
    }
}

// The same with load(i, v) filling v in place (for element types that are arrays).
template <typename T, typename Load, typename Store>
__device__ __forceinline__ void block_copy4_into(int total, Load load, Store store) {
    for (int i0 = threadIdx.x; i0 < total; i0 += 4 * blockDim.x) {
        T v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < total) load(i, v[u]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < total) store(i, v[u]);
        }
    }
}

// x pass forward: int32 charge grid -> half-complex rows
__global__ void k_fft_x_fwd(DevState st, const PmeSysDev* plans, const int4* items, int maxn) {
    extern __shared__ float2 sm[];
    const int4 it = items[blockIdx.x];
    const SysDesc& sd = st.sys[it.x];
    const FftPlanDev& pl = plans[it.x].px;
    const int K0 = pl.n, K0h = K0 / 2 + 1;
    const float iK0 = 1.f / (float)K0, iK0h = 1.f / (float)(K0 / 2 + 1);   // exact small quotients (div_small)
    const int stride = K0 | 1;
    float2* tw = sm;
    float2* A = sm + maxn;
    float2* B = A + FFT_XLINES * (maxn + 1);
    load_twiddles(tw, pl, st.pme_tw);
    const int nl = it.z;
    const int* g = st.pme_grid_fx + sd.pme_off + (size_t)it.y * K0;
    // the nl lines are contiguous: element i of the tile is g[i]
    block_copy4<int>(
        nl * K0, [&](int i) { return g[i]; },
        [&](int i, int v) {
            const int l = div_small(i, iK0), x = i - l * K0;
            A[l * stride + x] = make_float2((float)v * (float)(1.0 / GRID32_SCALE), 0.f);
        });
    __syncthreads();
    const float2* res = fft_lines(A, B, nl, stride, pl, tw, -1.f);
    float2* out = st.pme_cplx + sd.pme_coff + (size_t)it.y * K0h;
    for (int i = threadIdx.x; i < nl * K0h; i += blockDim.x) {
        const int l = div_small(i, iK0h), k = i - l * K0h;
        out[(size_t)l * K0h + k] = res[l * stride + k];
    }
}

// x pass inverse: half-complex rows -> real potential rows
__global__ void k_fft_x_inv(DevState st, const PmeSysDev* plans, const int4* items, int maxn) {
    extern __shared__ float2 sm[];
    const int4 it = items[blockIdx.x];
    const SysDesc& sd = st.sys[it.x];
    const FftPlanDev& pl = plans[it.x].px;
    const int K0 = pl.n, K0h = K0 / 2 + 1;
    const float iK0 = 1.f / (float)K0, iK0h = 1.f / (float)(K0 / 2 + 1);   // exact small quotients (div_small)
    const int stride = K0 | 1;
    float2* tw = sm;
    float2* A = sm + maxn;
    float2* B = A + FFT_XLINES * (maxn + 1);
    load_twiddles(tw, pl, st.pme_tw);
    const int nl = it.z;
    const float2* in = st.pme_cplx + sd.pme_coff + (size_t)it.y * K0h;
    block_copy4<float2>(
        nl * K0,
        [&](int i) {
            const int l = div_small(i, iK0), k = i - l * K0;
            float2 v;
            if (k < K0h) {
                v = in[(size_t)l * K0h + k];
            } else {
                v = in[(size_t)l * K0h + (K0 - k)];
                v.y = -v.y;  // Hermitian symmetry of a real signal
            }
            return v;
        },
        [&](int i, float2 v) {
            const int l = div_small(i, iK0), k = i - l * K0;
            A[l * stride + k] = v;
        });
    __syncthreads();
    const float2* res = fft_lines(A, B, nl, stride, pl, tw, 1.f);
    float* out = st.pme_real + sd.pme_off + (size_t)it.y * K0;
    for (int i = threadIdx.x; i < nl * K0; i += blockDim.x) {
        const int l = div_small(i, iK0), x = i - l * K0;
        out[(size_t)l * K0 + x] = res[l * stride + x].x;
    }
}

// y pass (either direction): tile of FFT_TX half-complex columns x all y, at one z
__global__ void k_fft_y(DevState st, const PmeSysDev* plans, const int4* items, float sigma, int maxn) {
    extern __shared__ float2 sm[];
    const int4 it = items[blockIdx.x];
    const SysDesc& sd = st.sys[it.x];
    const FftPlanDev& pl = plans[it.x].py;
    const int K0h = plans[it.x].px.n / 2 + 1, K1 = pl.n;
    const int stride = K1 | 1;
    float2* tw = sm;
    float2* A = sm + maxn;
    float2* B = A + FFT_TX * (maxn + 1);
    load_twiddles(tw, pl, st.pme_tw);
    const int x0 = it.y, z = it.z;
    const int tx = min(FFT_TX, K0h - x0);
    float2* g = st.pme_cplx + sd.pme_coff + (size_t)z * K1 * K0h + x0;
    block_copy4<float2>(
        K1 * FFT_TX,
        [&](int i) {
            const int y = i / FFT_TX, c = i - y * FFT_TX;
            return c < tx ? g[(size_t)y * K0h + c] : make_float2(0.f, 0.f);
        },
        [&](int i, float2 v) {
            const int y = i / FFT_TX, c = i - y * FFT_TX;
            A[c * stride + y] = v;
        });
    __syncthreads();
    const float2* res = fft_lines(A, B, FFT_TX, stride, pl, tw, sigma);
    for (int i = threadIdx.x; i < K1 * FFT_TX; i += blockDim.x) {
        const int y = i / FFT_TX, c = i - y * FFT_TX;
        if (c < tx) g[(size_t)y * K0h + c] = res[c * stride + y];
    }
}

// z pass: forward FFT along z, multiply by theta(k), inverse FFT along z.  The
// tile's theta values are loaded together with its grid values (one round of
// global-load latency for both) and wait in shared memory for the product.
__global__ void k_fft_z_conv(DevState st, const PmeSysDev* plans, const int4* items, int maxn) {
    extern __shared__ float2 sm[];
    const int4 it = items[blockIdx.x];
    const SysDesc& sd = st.sys[it.x];
    const FftPlanDev& pl = plans[it.x].pz;
    const int K0h = plans[it.x].px.n / 2 + 1, K1 = plans[it.x].py.n, K2 = pl.n;
    const int stride = K2 | 1;
    float2* tw = sm;
    float2* A = sm + maxn;
    float2* B = A + FFT_TX * (maxn + 1);
    float* T = reinterpret_cast<float*>(B + FFT_TX * (maxn + 1));   // theta, [z][c]
    load_twiddles(tw, pl, st.pme_tw);
    const int x0 = it.y, y = it.z;
    const int tx = min(FFT_TX, K0h - x0);
    const size_t plane = (size_t)K1 * K0h;
    float2* g = st.pme_cplx + sd.pme_coff + (size_t)y * K0h + x0;
    const float* th = st.pme_theta + sd.pme_coff + (size_t)y * K0h + x0;
    const int total = K2 * FFT_TX;
    for (int i0 = threadIdx.x; i0 < total; i0 += 4 * blockDim.x) {
        float2 v[4];
        float t[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * blockDim.x;
            const int z = i / FFT_TX, c = i - z * FFT_TX;
            const bool ok = i < total && c < tx;
            v[u] = ok ? g[z * plane + c] : make_float2(0.f, 0.f);
            t[u] = ok ? th[z * plane + c] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < total) {
                const int z = i / FFT_TX, c = i - z * FFT_TX;
                A[c * stride + z] = v[u];
                T[i] = t[u];
            }
        }
    }
    __syncthreads();
    float2* res = fft_lines(A, B, FFT_TX, stride, pl, tw, -1.f);
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        const int z = i / FFT_TX, c = i - z * FFT_TX;
        res[c * stride + z] = cscale(res[c * stride + z], T[i]);
    }
    __syncthreads();
    float2* other = res == A ? B : A;
    const float2* res2 = fft_lines(res, other, FFT_TX, stride, pl, tw, 1.f);
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        const int z = i / FFT_TX, c = i - z * FFT_TX;
        if (c < tx) g[z * plane + c] = res2[c * stride + z];
    }
}

// ------------------------------------------------------- plane-fused x+y
// One CTA per z-plane.  Forward: the plane's K1 real rows are packed two per
// complex line (row 2p + i row 2p+1), transformed along x, separated with the
// symmetry of real transforms (X_a[k] = (Z[k] + conj Z[-k]) / 2,
// X_b[k] = -i (Z[k] - conj Z[-k]) / 2) straight into y-lines, transformed along
// y and written as the half-complex plane.  Inverse: the reverse, ending with
// the two real rows of each line in its real and imaginary parts.
constexpr int FFT_XY_THREADS = 512;

__device__ __forceinline__ int xy_lines(int k1) { return (k1 + 1) / 2; }

__global__ void __launch_bounds__(FFT_XY_THREADS) k_fft_xy_fwd(DevState st, const PmeSysDev* plans, const int4* items,
                                                               int maxn, int buf) {
    extern __shared__ float2 sm[];
    const int4 it = items[blockIdx.x];
    const SysDesc& sd = st.sys[it.x];
    const FftPlanDev& plx = plans[it.x].px;
    const FftPlanDev& ply = plans[it.x].py;
    const int K0 = plx.n, K1 = ply.n, K0h = K0 / 2 + 1, P = xy_lines(K1), z = it.y;
    const float iK0 = 1.f / (float)K0, iK0h = 1.f / (float)(K0 / 2 + 1);   // exact small quotients (div_small)
    float2* twx = sm;
    float2* twy = sm + maxn;
    float2* A = sm + 2 * maxn;
    float2* B = A + buf;
    load_twiddles(twx, plx, st.pme_tw);
    load_twiddles(twy, ply, st.pme_tw);
    const int* g = st.pme_grid_fx + sd.pme_off + (size_t)K0 * K1 * z;
    const int sx = K0 + 1, sy = K1 + 1;
    constexpr float isc = (float)(1.0 / GRID32_SCALE);
    if ((K0 & 3) == 0 && (sd.pme_off & 3) == 0) {
        // rows of a multiple of four nodes from a 16-byte aligned plane: four x
        // nodes of both rows of a line per element
        const int K0q = K0 >> 2;
        const float iK0q = 1.f / (float)K0q;
        block_copy4_into<int4[2]>(
            P * K0q,
            [&](int i, int4 (&v)[2]) {
                const int pl = div_small(i, iK0q), x = 4 * (i - pl * K0q);
                const int ya = 2 * pl, yb = ya + 1;
                v[0] = *reinterpret_cast<const int4*>(g + (size_t)ya * K0 + x);
                v[1] = yb < K1 ? *reinterpret_cast<const int4*>(g + (size_t)yb * K0 + x) : make_int4(0, 0, 0, 0);
            },
            [&](int i, const int4 (&v)[2]) {
                const int pl = div_small(i, iK0q), x = 4 * (i - pl * K0q);
                float2* a = A + pl * sx + x;
                a[0] = make_float2((float)v[0].x * isc, (float)v[1].x * isc);
                a[1] = make_float2((float)v[0].y * isc, (float)v[1].y * isc);
                a[2] = make_float2((float)v[0].z * isc, (float)v[1].z * isc);
                a[3] = make_float2((float)v[0].w * isc, (float)v[1].w * isc);
            });
    } else {
        block_copy4<float2>(
            P * K0,
            [&](int i) {
                const int pl = div_small(i, iK0), x = i - pl * K0;
                const int ya = 2 * pl, yb = ya + 1;
                const float a = (float)g[(size_t)ya * K0 + x] * isc;
                const float b = yb < K1 ? (float)g[(size_t)yb * K0 + x] * isc : 0.f;
                return make_float2(a, b);
            },
            [&](int i, float2 v) {
                const int pl = div_small(i, iK0), x = i - pl * K0;
                A[pl * sx + x] = v;
            });
    }
    __syncthreads();
    const float2* res = fft_lines(A, B, P, sx, plx, twx, -1.f);
    float2* yl = res == A ? B : A;
    for (int i = threadIdx.x; i < P * K0h; i += blockDim.x) {
        const int pl = div_small(i, iK0h), k = i - pl * K0h;
        const float2 Z = res[pl * sx + k];
        const float2 Zm = res[pl * sx + (k == 0 ? 0 : K0 - k)];
        yl[k * sy + 2 * pl] = make_float2(0.5f * (Z.x + Zm.x), 0.5f * (Z.y - Zm.y));
        if (2 * pl + 1 < K1) yl[k * sy + 2 * pl + 1] = make_float2(0.5f * (Z.y + Zm.y), -0.5f * (Z.x - Zm.x));
    }
    __syncthreads();
    const float2* out = fft_lines(yl, const_cast<float2*>(res), K0h, sy, ply, twy, -1.f);
    float2* gc = st.pme_cplx + sd.pme_coff + (size_t)K0h * K1 * z;
    for (int i = threadIdx.x; i < K1 * K0h; i += blockDim.x) {
        const int y = div_small(i, iK0h), x = i - y * K0h;
        gc[(size_t)y * K0h + x] = out[x * sy + y];
    }
}

__global__ void __launch_bounds__(FFT_XY_THREADS) k_fft_xy_inv(DevState st, const PmeSysDev* plans, const int4* items,
                                                               int maxn, int buf) {
    extern __shared__ float2 sm[];
    const int4 it = items[blockIdx.x];
    const SysDesc& sd = st.sys[it.x];
    const FftPlanDev& plx = plans[it.x].px;
    const FftPlanDev& ply = plans[it.x].py;
    const int K0 = plx.n, K1 = ply.n, K0h = K0 / 2 + 1, P = xy_lines(K1), z = it.y;
    const float iK0 = 1.f / (float)K0, iK0h = 1.f / (float)(K0 / 2 + 1);   // exact small quotients (div_small)
    float2* twx = sm;
    float2* twy = sm + maxn;
    float2* A = sm + 2 * maxn;
    float2* B = A + buf;
    load_twiddles(twx, plx, st.pme_tw);
    load_twiddles(twy, ply, st.pme_tw);
    const float2* gc = st.pme_cplx + sd.pme_coff + (size_t)K0h * K1 * z;
    const int sx = K0 + 1, sy = K1 + 1;
    block_copy4<float2>(
        K1 * K0h, [&](int i) { return gc[i]; },
        [&](int i, float2 v) {
            const int y = div_small(i, iK0h), x = i - y * K0h;
            A[x * sy + y] = v;
        });
    __syncthreads();
    const float2* res = fft_lines(A, B, K0h, sy, ply, twy, 1.f);
    float2* xl = res == A ? B : A;
    // full spectra of rows 2p and 2p+1 (Hermitian symmetry beyond K0h), packed as a + i b
    for (int i = threadIdx.x; i < P * K0; i += blockDim.x) {
        const int pl = div_small(i, iK0), k = i - pl * K0;
        const int ya = 2 * pl, yb = ya + 1;
        float2 a, b = make_float2(0.f, 0.f);
        if (k < K0h) {
            a = res[k * sy + ya];
            if (yb < K1) b = res[k * sy + yb];
        } else {
            a = res[(K0 - k) * sy + ya];
            a.y = -a.y;
            if (yb < K1) {
                b = res[(K0 - k) * sy + yb];
                b.y = -b.y;
            }
        }
        xl[pl * sx + k] = make_float2(a.x - b.y, a.y + b.x);
    }
    __syncthreads();
    const float2* out = fft_lines(xl, const_cast<float2*>(res), P, sx, plx, twx, 1.f);
    float* gr = st.pme_real + sd.pme_off + (size_t)K0 * K1 * z;
    if ((K0 & 3) == 0 && (sd.pme_off & 3) == 0) {
        // four x nodes per store (16-byte aligned rows)
        const int K0q = K0 >> 2;
        const float iK0q = 1.f / (float)K0q;
        for (int i = threadIdx.x; i < K1 * K0q; i += blockDim.x) {
            const int y = div_small(i, iK0q), x = 4 * (i - y * K0q);
            const float2* o = out + (y >> 1) * sx + x;
            const float2 v0 = o[0], v1 = o[1], v2 = o[2], v3 = o[3];
            *reinterpret_cast<float4*>(gr + (size_t)y * K0 + x) =
                (y & 1) ? make_float4(v0.y, v1.y, v2.y, v3.y) : make_float4(v0.x, v1.x, v2.x, v3.x);
        }
    } else {
        for (int i = threadIdx.x; i < K1 * K0; i += blockDim.x) {
            const int y = div_small(i, iK0), x = i - y * K0;
            const float2 v = out[(y >> 1) * sx + x];
            gr[(size_t)y * K0 + x] = (y & 1) ? v.y : v.x;
        }
    }
}

int pme_xy_buffer(int k0, int k1) {
    const int k0h = k0 / 2 + 1, P = (k1 + 1) / 2;
    const int buf = std::max(P * (k0 + 1), k0h * (k1 + 1));
    // two ping-pong buffers and two twiddle tables within ~200 KB
    if ((size_t)(2 * buf + 2 * FFT_MAXN) * sizeof(float2) > 200 * 1024) return 0;
    return (buf + 1) & ~1;
}

// ------------------------------------------------------------------ gather
// Four threads per atom (adjacent lanes), one z-plane of the stencil each: the
// first shuffle pairs planes 0 and 1, and 2 and 3, the second gives
// (p0 + p1) + (p2 + p3).
// ONE: a single system, whose descriptor sd1 comes as a kernel argument instead
// of a dependent load through the cluster's system index.
template <bool ENERGY, bool FD, bool ONE>
__global__ void k_gather(DevState st, const SysDesc sd1) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = t >> 2, quarter = t & 3;
    double e = 0.0;
    int sysi = -1;
    float q = 0.f, phi = 0.f, gx = 0.f, gy = 0.f, gz = 0.f, sc0 = 0.f, sc1 = 0.f, sc2 = 0.f;
    if (s < st.n_slots) {
        const float4 p = st.xyzq[s];
        const int sy = ONE ? 0 : st.cluster_sys[s / CLUSTER];
        const SysDesc& sd = ONE ? sd1 : st.sys[sy];
        if (p.w != 0.f && st.orig[s] >= 0 && sd.pme_n[0] != 0) {
            sysi = sy;
            q = p.w;
            const int K0 = sd.pme_n[0], K1 = sd.pme_n[1], K2 = sd.pme_n[2];
            int b0, b1, b2;
            float f0, f1, f2;
            grid_coord(p.x, sd.pme_inv_h[0], K0, b0, f0);
            grid_coord(p.y, sd.pme_inv_h[1], K1, b1, f1);
            grid_coord(p.z, sd.pme_inv_h[2], K2, b2, f2);
            float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
            bspline4(f0, wx);
            bspline4(f1, wy);
            bspline4(f2, wz);
            bspline4_d(f0, dx);
            bspline4_d(f1, dy);
            bspline4_d(f2, dz);
            const float* g = st.pme_real + sd.pme_off;
            int ix[4], ixp[4], ixm[4], iy[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                ix[a] = wrap1(b0 - 1 + a, K0);
                ixp[a] = wrap1(b0 + a, K0);
                ixm[a] = wrap1(b0 - 2 + a, K0);
                iy[a] = wrap1(b1 - 1 + a, K1);
            }
            // this lane's plane of the stencil
            {
                const int c = quarter;
                const int z = wrap1(b2 - 1 + c, K2);
                const float wzc = pick4(wz, c), dzc = pick4(dz, c);
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int y = iy[b];
                    const float* row = g + (size_t)K0 * (y + (size_t)K1 * z);
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const float v = row[ix[a]];
                        const float w = wx[a] * wy[b] * wzc;
                        phi += w * v;
                        if (FD) {
                            const int yp = wrap1(y + 1, K1), ym = wrap1(y - 1, K1);
                            const int zp = wrap1(z + 1, K2), zm = wrap1(z - 1, K2);
                            gx += w * (row[ixp[a]] - row[ixm[a]]);
                            gy += w * (g[(size_t)K0 * (yp + (size_t)K1 * z) + ix[a]] -
                                       g[(size_t)K0 * (ym + (size_t)K1 * z) + ix[a]]);
                            gz += w * (g[(size_t)K0 * (y + (size_t)K1 * zp) + ix[a]] -
                                       g[(size_t)K0 * (y + (size_t)K1 * zm) + ix[a]]);
                        } else {
                            gx += dx[a] * wy[b] * wzc * v;
                            gy += wx[a] * dy[b] * wzc * v;
                            gz += wx[a] * wy[b] * dzc * v;
                        }
                    }
                }
            }
            sc0 = FD ? 0.5f * sd.pme_inv_h[0] : sd.pme_inv_h[0];
            sc1 = FD ? 0.5f * sd.pme_inv_h[1] : sd.pme_inv_h[1];
            sc2 = FD ? 0.5f * sd.pme_inv_h[2] : sd.pme_inv_h[2];
        }
    }
    // (p0 + p1) + (p2 + p3)
    phi += __shfl_xor_sync(0xffffffffu, phi, 1);
    gx += __shfl_xor_sync(0xffffffffu, gx, 1);
    gy += __shfl_xor_sync(0xffffffffu, gy, 1);
    gz += __shfl_xor_sync(0xffffffffu, gz, 1);
    phi += __shfl_xor_sync(0xffffffffu, phi, 2);
    gx += __shfl_xor_sync(0xffffffffu, gx, 2);
    gy += __shfl_xor_sync(0xffffffffu, gy, 2);
    gz += __shfl_xor_sync(0xffffffffu, gz, 2);
    if (sysi >= 0 && quarter == 0) {
        atomic_add_fixed(st.fx + s, to_fixed(-q * gx * sc0, FORCE_SCALE));
        atomic_add_fixed(st.fy + s, to_fixed(-q * gy * sc1, FORCE_SCALE));
        atomic_add_fixed(st.fz + s, to_fixed(-q * gz * sc2, FORCE_SCALE));
        if (ENERGY) {
            e = 0.5 * (double)q * (double)phi;
            // the atom's reciprocal energy and its share of the Ewald self term
            if (st.atom_energy) {
                const SysDesc& sd = ONE ? sd1 : st.sys[sysi];
                const double self = sd.self_per_charge ? (double)sd.self_coef : (double)sd.self_coef * q * q;
                add_atom_energy(st.epot, s, e + self);
            }
        }
    }
    if (ENERGY) add_energy_fixed(st.energy, quarter == 0 ? sysi : -1, e, E_RECIP);
}

// ------------------------------------------------------------------ driver
static size_t fft_smem_bytes(int lines, int maxn) {
    return (size_t)(maxn + 2 * lines * (maxn + 1)) * sizeof(float2);
}
// the z pass also holds its tile's theta values
static size_t zconv_smem_bytes(int maxn) {
    return fft_smem_bytes(FFT_TX, maxn) + (size_t)FFT_TX * maxn * sizeof(float);
}

int launch_pme(const DevState& st, const PmePlan& plan, bool energy, cudaStream_t s) {
    if (plan.n_items_x == 0) return 0;
    const PmeSysDev* plans = reinterpret_cast<const PmeSysDev*>(plan.sys_plans);
    const int TB = 256;
    const int mx = plan.max_n;
    const size_t sx = fft_smem_bytes(FFT_XLINES, mx), sy = fft_smem_bytes(FFT_TX, mx);
    cudaMemsetAsync(st.pme_grid_fx, 0, sizeof(int) * (size_t)st.pme_total_real, s);
    const int g4 = (int)(((long long)st.n_slots * 4 + TB - 1) / TB);
    if (plan.n_items_spread > 0)
        k_spread_tiles<<<plan.n_items_spread, 256, (size_t)plan.spread_box * sizeof(int), s>>>(
            st, plan.items_spread, plan.spread_geo);
    else
        k_spread<<<g4, TB, 0, s>>>(st);
    int n = 7;
    if (plan.n_items_xy > 0) {
        const size_t sxy = (size_t)(2 * mx + 2 * plan.xy_buf) * sizeof(float2);
        k_fft_xy_fwd<<<plan.n_items_xy, FFT_XY_THREADS, sxy, s>>>(st, plans, plan.items_xy, mx, plan.xy_buf);
        k_fft_z_conv<<<plan.n_items_z, FFT_YZ_THREADS, zconv_smem_bytes(mx), s>>>(st, plans, plan.items_z, mx);
        k_fft_xy_inv<<<plan.n_items_xy, FFT_XY_THREADS, sxy, s>>>(st, plans, plan.items_xy, mx, plan.xy_buf);
        n = 5;
    } else {
        k_fft_x_fwd<<<plan.n_items_x, 256, sx, s>>>(st, plans, plan.items_x, mx);
        k_fft_y<<<plan.n_items_y, FFT_YZ_THREADS, sy, s>>>(st, plans, plan.items_y, -1.f, mx);
        k_fft_z_conv<<<plan.n_items_z, FFT_YZ_THREADS, zconv_smem_bytes(mx), s>>>(st, plans, plan.items_z, mx);
        k_fft_y<<<plan.n_items_y, FFT_YZ_THREADS, sy, s>>>(st, plans, plan.items_y, 1.f, mx);
        k_fft_x_inv<<<plan.n_items_x, 256, sx, s>>>(st, plans, plan.items_x, mx);
    }
    const SysDesc& sd1 = plan.sys0;
    const int g1 = (int)(((long long)st.n_slots * 4 + TB - 1) / TB);   // gather: four threads per slot
    if (plan.n_sys == 1) {
        if (plan.ref_gather) {
            if (energy) k_gather<true, true, true><<<g1, TB, 0, s>>>(st, sd1);
            else k_gather<false, true, true><<<g1, TB, 0, s>>>(st, sd1);
        } else {
            if (energy) k_gather<true, false, true><<<g1, TB, 0, s>>>(st, sd1);
            else k_gather<false, false, true><<<g1, TB, 0, s>>>(st, sd1);
        }
    } else if (plan.ref_gather) {
        if (energy) k_gather<true, true, false><<<g1, TB, 0, s>>>(st, sd1);
        else k_gather<false, true, false><<<g1, TB, 0, s>>>(st, sd1);
    } else {
        if (energy) k_gather<true, false, false><<<g1, TB, 0, s>>>(st, sd1);
        else k_gather<false, false, false><<<g1, TB, 0, s>>>(st, sd1);
    }
    return n;
}

// Host helper: radix plan for an FFT length (8s first, then 4s, 2, 3, 5: fewer
// stages mean fewer shared-memory passes and barriers).
bool make_fft_plan(int n, FftPlanDev* out) {
    if (n < 2 || n > FFT_MAXN) return false;
    out->n = n;
    out->nrad = 0;
    out->tw_off = -1;
    int m = n;
    while (m % 8 == 0) {
        out->rad[out->nrad++] = 8;
        m /= 8;
    }
    while (m % 4 == 0) {
        out->rad[out->nrad++] = 4;
        m /= 4;
    }
    for (int p : {2, 3, 5}) {
        while (m % p == 0) {
            if (out->nrad >= 12) return false;
            out->rad[out->nrad++] = p;
            m /= p;
        }
    }
    return m == 1;
}

size_t pme_sys_dev_size() { return sizeof(PmeSysDev); }

bool fill_pme_sys_dev(void* dst, int kx, int ky, int kz) {
    PmeSysDev* d = reinterpret_cast<PmeSysDev*>(dst);
    return make_fft_plan(kx, &d->px) && make_fft_plan(ky, &d->py) && make_fft_plan(kz, &d->pz);
}

void set_pme_sys_twiddles(void* dst, int offx, int offy, int offz) {
    PmeSysDev* d = reinterpret_cast<PmeSysDev*>(dst);
    d->px.tw_off = offx;
    d->py.tw_off = offy;
    d->pz.tw_off = offz;
}

// The attribute belongs to the kernel on one device and is shared by every
// engine on that device: it only ever grows there, so an engine with small grids
// cannot shrink the room another engine relies on.
void pme_set_smem_limits(int maxn, int xy_buf) {
    static std::mutex mu;
    static int largest_xy[64] = {}, largest[64] = {};
    static bool spread_attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    dev &= 63;
    std::lock_guard<std::mutex> lock(mu);
    if (!spread_attr[dev]) {
        cudaFuncSetAttribute(k_spread_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             PME_SPREAD_MAX_BOX * (int)sizeof(int));
        spread_attr[dev] = true;
    }
    if (xy_buf > largest_xy[dev]) {
        largest_xy[dev] = xy_buf;
        const int b = (int)((size_t)(2 * FFT_MAXN + 2 * xy_buf) * sizeof(float2));
        cudaFuncSetAttribute(k_fft_xy_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
        cudaFuncSetAttribute(k_fft_xy_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    }
    if (maxn <= largest[dev]) return;
    largest[dev] = maxn;
    const int by = (int)fft_smem_bytes(FFT_TX, maxn), bx = (int)fft_smem_bytes(FFT_XLINES, maxn);
    cudaFuncSetAttribute(k_fft_y, cudaFuncAttributeMaxDynamicSharedMemorySize, by);
    cudaFuncSetAttribute(k_fft_z_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zconv_smem_bytes(maxn));
    cudaFuncSetAttribute(k_fft_x_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, bx);
    cudaFuncSetAttribute(k_fft_x_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, bx);
}

}  // namespace lima

namespace lima {

// ===================================================================== no-alloc
// Reciprocal-space PME for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc: a plug-in inside an
// application that owns every device allocation through its own pool (its own
// cudaMalloc would bypass the host's accounting), or a real-time loop that must
// not allocate after start-up (cudaMalloc may synchronise the device).  For them lima_pme_recip_noalloc
// computes the same reciprocal-space forces and energy as the engine's PME
// stage, using the static scratch array below instead of allocated grids.
//
// Limits: at most NOALLOC_MAX_POINTS real grid points (64^3) and at most
// NOALLOC_MAX_DIM points per dimension.  Every GPU that loads this library
// holds NOALLOC_SCRATCH_BYTES (~5 MB) of static device memory until the
// process exits.  All calls share the array and it keeps the last call's
// contents; each call clears what must start at zero.  Calls whose work
// overlaps on the GPU (other streams, other host threads) race on the array.
namespace {
constexpr int NOALLOC_MAX_POINTS = 64 * 64 * 64;
constexpr int NOALLOC_MAX_DIM = 128;
constexpr size_t NOALLOC_HALF_POINTS = (size_t)NOALLOC_MAX_POINTS * 5 / 8;  // >= (K0/2+1)K1K2 for K0 >= 8
constexpr size_t NOALLOC_OFF_REAL = (size_t)NOALLOC_MAX_POINTS * sizeof(long long);
constexpr size_t NOALLOC_OFF_CPLX = NOALLOC_OFF_REAL + (size_t)NOALLOC_MAX_POINTS * sizeof(float);
constexpr size_t NOALLOC_OFF_THETA = NOALLOC_OFF_CPLX + NOALLOC_HALF_POINTS * sizeof(float2);
constexpr size_t NOALLOC_OFF_ENERGY = NOALLOC_OFF_THETA + NOALLOC_HALF_POINTS * sizeof(float);
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_OFF_ENERGY + 256;
}  // namespace

static __device__ __align__(256) unsigned char g_pme_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

struct NaGrid {
    int n[3];
    float inv_h[3];
    double box[3];
    double kappa;
    FftPlanDev px, py, pz;
};

__device__ __forceinline__ long long* na_grid(unsigned char* s) { return reinterpret_cast<long long*>(s); }
__device__ __forceinline__ float* na_real(unsigned char* s) { return reinterpret_cast<float*>(s + NOALLOC_OFF_REAL); }
__device__ __forceinline__ float2* na_cplx(unsigned char* s) { return reinterpret_cast<float2*>(s + NOALLOC_OFF_CPLX); }
__device__ __forceinline__ float* na_theta(unsigned char* s) { return reinterpret_cast<float*>(s + NOALLOC_OFF_THETA); }
__device__ __forceinline__ long long* na_energy(unsigned char* s) {
    return reinterpret_cast<long long*>(s + NOALLOC_OFF_ENERGY);
}

// zero the charge grid and the energy accumulator; influence function (SPME,
// B-spline moduli of the centred order-4 weights, 1/N folded in) in FP64
__global__ void k_na_prepare(unsigned char* scratch, NaGrid g) {
    const int K0 = g.n[0], K1 = g.n[1], K2 = g.n[2], K0h = K0 / 2 + 1;
    const int N = K0 * K1 * K2, Nh = K0h * K1 * K2;
    long long* grid = na_grid(scratch);
    float* theta = na_theta(scratch);
    const double ke = 8.9875517873681764e9 / 1e-9 / 6.02214076e23 * 1000.0 * 1000.0;
    const double pi = 3.14159265358979323846;
    const double V = g.box[0] * g.box[1] * g.box[2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < max(N, Nh); i += gridDim.x * blockDim.x) {
        if (i < N) grid[i] = 0;
        if (i < Nh) {
            const int x = i % K0h, y = (i / K0h) % K1, z = i / (K0h * K1);
            const int m[3] = {x, y <= K1 / 2 ? y : y - K1, z <= K2 / 2 ? z : z - K2};
            double t = 0.0;
            if (m[0] != 0 || m[1] != 0 || m[2] != 0) {
                double k2 = 0.0, B = 1.0;
                for (int d = 0; d < 3; ++d) {
                    const double kv = 2.0 * pi * m[d] / g.box[d];
                    k2 += kv * kv;
                    const double b = 2.0 / 3.0 + cos(2.0 * pi * m[d] / g.n[d]) / 3.0;
                    B *= b * b;
                }
                t = ke * 4.0 * pi / k2 * exp(-k2 / (4.0 * g.kappa * g.kappa)) / V / B;
            }
            theta[i] = (float)t;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *na_energy(scratch) = 0;
}

__global__ void k_na_spread(const float4* __restrict__ xyzq, int n, unsigned char* scratch, NaGrid g) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const float4 p = xyzq[a];
    if (p.w == 0.f) return;
    const int K0 = g.n[0], K1 = g.n[1], K2 = g.n[2];
    int b0, b1, b2;
    float f0, f1, f2;
    grid_coord(p.x, g.inv_h[0], K0, b0, f0);
    grid_coord(p.y, g.inv_h[1], K1, b1, f1);
    grid_coord(p.z, g.inv_h[2], K2, b2, f2);
    float wx[4], wy[4], wz[4];
    bspline4(f0, wx);
    bspline4(f1, wy);
    bspline4(f2, wz);
    long long* grid = na_grid(scratch);
    int ix[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) ix[k] = wrapk(b0 - 1 + k, K0);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int z = wrapk(b2 - 1 + c, K2);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int y = wrapk(b1 - 1 + b, K1);
            const float qyz = p.w * wy[b] * wz[c];
            long long* row = grid + (size_t)K0 * (y + (size_t)K1 * z);
#pragma unroll
            for (int k = 0; k < 4; ++k) atomic_add_fixed(row + ix[k], to_fixed(qyz * wx[k], GRID_SCALE));
        }
    }
}

// x pass forward: block b handles lines [8b, 8b+8) of the K1*K2 lines
__global__ void k_na_fft_x_fwd(unsigned char* scratch, NaGrid g) {
    extern __shared__ float2 sm[];
    const FftPlanDev& pl = g.px;
    const int K0 = pl.n, K0h = K0 / 2 + 1, stride = K0 | 1, maxn = NOALLOC_MAX_DIM;
    float2* tw = sm;
    float2* A = sm + maxn;
    float2* B = A + FFT_XLINES * (maxn + 1);
    make_twiddles(tw, K0);
    const int line0 = blockIdx.x * FFT_XLINES;
    const int nl = min(FFT_XLINES, g.n[1] * g.n[2] - line0);
    long long* grid = na_grid(scratch) + (size_t)line0 * K0;
    for (int i = threadIdx.x; i < nl * K0; i += blockDim.x) {
        const int l = i / K0, x = i - l * K0;
        A[l * stride + x] = make_float2((float)((double)grid[(size_t)l * K0 + x] * (1.0 / GRID_SCALE)), 0.f);
    }
    __syncthreads();
    const float2* res = fft_lines(A, B, nl, stride, pl, tw, -1.f);
    float2* out = na_cplx(scratch) + (size_t)line0 * K0h;
    for (int i = threadIdx.x; i < nl * K0h; i += blockDim.x) {
        const int l = i / K0h, k = i - l * K0h;
        out[(size_t)l * K0h + k] = res[l * stride + k];
    }
}

__global__ void k_na_fft_x_inv(unsigned char* scratch, NaGrid g) {
    extern __shared__ float2 sm[];
    const FftPlanDev& pl = g.px;
    const int K0 = pl.n, K0h = K0 / 2 + 1, stride = K0 | 1, maxn = NOALLOC_MAX_DIM;
    float2* tw = sm;
    float2* A = sm + maxn;
    float2* B = A + FFT_XLINES * (maxn + 1);
    make_twiddles(tw, K0);
    const int line0 = blockIdx.x * FFT_XLINES;
    const int nl = min(FFT_XLINES, g.n[1] * g.n[2] - line0);
    const float2* in = na_cplx(scratch) + (size_t)line0 * K0h;
    for (int i = threadIdx.x; i < nl * K0; i += blockDim.x) {
        const int l = i / K0, k = i - l * K0;
        float2 v;
        if (k < K0h) {
            v = in[(size_t)l * K0h + k];
        } else {
            v = in[(size_t)l * K0h + (K0 - k)];
            v.y = -v.y;
        }
        A[l * stride + k] = v;
    }
    __syncthreads();
    const float2* res = fft_lines(A, B, nl, stride, pl, tw, 1.f);
    float* out = na_real(scratch) + (size_t)line0 * K0;
    for (int i = threadIdx.x; i < nl * K0; i += blockDim.x) {
        const int l = i / K0, x = i - l * K0;
        out[(size_t)l * K0 + x] = res[l * stride + x].x;
    }
}

// y pass: block (x-tile, z)
__global__ void k_na_fft_y(unsigned char* scratch, NaGrid g, float sigma) {
    extern __shared__ float2 sm[];
    const FftPlanDev& pl = g.py;
    const int K0h = g.n[0] / 2 + 1, K1 = pl.n, stride = K1 | 1, maxn = NOALLOC_MAX_DIM;
    float2* tw = sm;
    float2* A = sm + maxn;
    float2* B = A + FFT_TX * (maxn + 1);
    make_twiddles(tw, K1);
    const int ntx = (K0h + FFT_TX - 1) / FFT_TX;
    const int x0 = (blockIdx.x % ntx) * FFT_TX, z = blockIdx.x / ntx;
    const int tx = min(FFT_TX, K0h - x0);
    float2* gp = na_cplx(scratch) + (size_t)z * K1 * K0h + x0;
    for (int i = threadIdx.x; i < K1 * FFT_TX; i += blockDim.x) {
        const int y = i / FFT_TX, c = i - y * FFT_TX;
        A[c * stride + y] = c < tx ? gp[(size_t)y * K0h + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const float2* res = fft_lines(A, B, FFT_TX, stride, pl, tw, sigma);
    for (int i = threadIdx.x; i < K1 * FFT_TX; i += blockDim.x) {
        const int y = i / FFT_TX, c = i - y * FFT_TX;
        if (c < tx) gp[(size_t)y * K0h + c] = res[c * stride + y];
    }
}

// z pass: block (x-tile, y); forward FFT, x theta, inverse FFT
__global__ void k_na_fft_z_conv(unsigned char* scratch, NaGrid g) {
    extern __shared__ float2 sm[];
    const FftPlanDev& pl = g.pz;
    const int K0h = g.n[0] / 2 + 1, K1 = g.n[1], K2 = pl.n, stride = K2 | 1, maxn = NOALLOC_MAX_DIM;
    float2* tw = sm;
    float2* A = sm + maxn;
    float2* B = A + FFT_TX * (maxn + 1);
    make_twiddles(tw, K2);
    const int ntx = (K0h + FFT_TX - 1) / FFT_TX;
    const int x0 = (blockIdx.x % ntx) * FFT_TX, y = blockIdx.x / ntx;
    const int tx = min(FFT_TX, K0h - x0);
    const size_t plane = (size_t)K1 * K0h;
    float2* gp = na_cplx(scratch) + (size_t)y * K0h + x0;
    const float* th = na_theta(scratch) + (size_t)y * K0h + x0;
    for (int i = threadIdx.x; i < K2 * FFT_TX; i += blockDim.x) {
        const int z = i / FFT_TX, c = i - z * FFT_TX;
        A[c * stride + z] = c < tx ? gp[z * plane + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* res = fft_lines(A, B, FFT_TX, stride, pl, tw, -1.f);
    for (int i = threadIdx.x; i < K2 * FFT_TX; i += blockDim.x) {
        const int z = i / FFT_TX, c = i - z * FFT_TX;
        const float t = c < tx ? th[z * plane + c] : 0.f;
        res[c * stride + z] = cscale(res[c * stride + z], t);
    }
    __syncthreads();
    float2* other = res == A ? B : A;
    const float2* res2 = fft_lines(res, other, FFT_TX, stride, pl, tw, 1.f);
    for (int i = threadIdx.x; i < K2 * FFT_TX; i += blockDim.x) {
        const int z = i / FFT_TX, c = i - z * FFT_TX;
        if (c < tx) gp[z * plane + c] = res2[c * stride + z];
    }
}

// analytic-derivative gather; forces are rounded through the same int64 fixed
// point the engine accumulates in, so both paths return identical values
__global__ void k_na_gather(const float4* __restrict__ xyzq, int n, unsigned char* scratch, NaGrid g,
                            double* __restrict__ forces) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (a < n) {
        const float4 p = xyzq[a];
        float fx = 0.f, fy = 0.f, fz = 0.f;
        if (p.w != 0.f) {
            const int K0 = g.n[0], K1 = g.n[1], K2 = g.n[2];
            int b0, b1, b2;
            float f0, f1, f2;
            grid_coord(p.x, g.inv_h[0], K0, b0, f0);
            grid_coord(p.y, g.inv_h[1], K1, b1, f1);
            grid_coord(p.z, g.inv_h[2], K2, b2, f2);
            float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
            bspline4(f0, wx);
            bspline4(f1, wy);
            bspline4(f2, wz);
            bspline4_d(f0, dx);
            bspline4_d(f1, dy);
            bspline4_d(f2, dz);
            const float* gr = na_real(scratch);
            int ix[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) ix[k] = wrapk(b0 - 1 + k, K0);
            float phi = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int z = wrapk(b2 - 1 + c, K2);
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int y = wrapk(b1 - 1 + b, K1);
                    const float* row = gr + (size_t)K0 * (y + (size_t)K1 * z);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float v = row[ix[k]];
                        phi += wx[k] * wy[b] * wz[c] * v;
                        gx += dx[k] * wy[b] * wz[c] * v;
                        gy += wx[k] * dy[b] * wz[c] * v;
                        gz += wx[k] * wy[b] * dz[c] * v;
                    }
                }
            }
            fx = -p.w * gx * g.inv_h[0];
            fy = -p.w * gy * g.inv_h[1];
            fz = -p.w * gz * g.inv_h[2];
            e = 0.5 * (double)p.w * (double)phi;
        }
        const double inv = 1.0 / FORCE_SCALE;
        forces[3 * a] = (double)to_fixed(fx, FORCE_SCALE) * inv;
        forces[3 * a + 1] = (double)to_fixed(fy, FORCE_SCALE) * inv;
        forces[3 * a + 2] = (double)to_fixed(fz, FORCE_SCALE) * inv;
    }
    add_energy_fixed(na_energy(scratch), a < n ? 0 : -1, e, 0);
}

__global__ void k_na_finish(unsigned char* scratch, double* energy) {
    *energy = (double)*na_energy(scratch) / ENERGY_SCALE;
}

namespace {
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[64] = {};
unsigned long long g_noalloc_ctx[64] = {};   // context id the cached address belongs to

// Unique id of the calling thread's current context (0 if the driver cannot
// tell).  The static array's address belongs to one context: after a
// cudaDeviceReset the runtime loads the module into a new context, so the
// cached address is refreshed whenever this id changes.  The driver entry
// points are fetched through the runtime, so the library needs no link
// against libcuda.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        looked_up = true;
    }
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
    return 0;
}
}  // namespace

}  // namespace lima

extern "C" int lima_pme_recip_noalloc(const float* d_xyzq, int n_atoms, double lx, double ly, double lz,
                                      int kx, int ky, int kz, double kappa, double* d_forces,
                                      double* d_energy, void* stream) {
    using namespace lima;
    if (n_atoms < 0 || (n_atoms > 0 && (!d_xyzq || !d_forces)) || !d_energy) return LIMA_ERR_INVALID_ARG;
    if (!(lx > 0.0 && ly > 0.0 && lz > 0.0) || !(kappa > 0.0)) return LIMA_ERR_INVALID_ARG;
    const int K[3] = {kx, ky, kz};
    for (int d = 0; d < 3; ++d)
        if (K[d] < 8) return LIMA_ERR_INVALID_ARG;
    if (kx > NOALLOC_MAX_DIM || ky > NOALLOC_MAX_DIM || kz > NOALLOC_MAX_DIM ||
        (long long)kx * ky * kz > NOALLOC_MAX_POINTS)
        return LIMA_ERR_OVERFLOW;  // beyond the static scratch array
    NaGrid g{};
    if (!make_fft_plan(kx, &g.px) || !make_fft_plan(ky, &g.py) || !make_fft_plan(kz, &g.pz))
        return LIMA_ERR_UNSUPPORTED;  // grid dimensions must factor into 2, 3 and 5
    const double L[3] = {lx, ly, lz};
    for (int d = 0; d < 3; ++d) {
        g.n[d] = K[d];
        g.box[d] = L[d];
        g.inv_h[d] = (float)(K[d] / L[d]);
    }
    g.kappa = kappa;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LIMA_ERR_NO_DEVICE;
    void* scratch = nullptr;
    {
        // set-up once per device (and again if the device's context changed):
        // the device address of the static array
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        // (no context yet reads as id 0; the lookup below creates the primary
        // context, and the next call refreshes the cache once under its id)
        const unsigned long long ctx = current_context_id();
        if (!g_noalloc_ptr[dev] || ctx != g_noalloc_ctx[dev]) {
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_pme_noalloc_scratch) != cudaSuccess || !ptr) return LIMA_ERR_CUDA;
            g_noalloc_ptr[dev] = ptr;
            g_noalloc_ctx[dev] = ctx;
        }
        scratch = g_noalloc_ptr[dev];
    }
    unsigned char* sp = static_cast<unsigned char*>(scratch);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int K0h = kx / 2 + 1;
    const int ntx = (K0h + FFT_TX - 1) / FFT_TX;
    const size_t sx = fft_smem_bytes(FFT_XLINES, NOALLOC_MAX_DIM), sy = fft_smem_bytes(FFT_TX, NOALLOC_MAX_DIM);
    k_na_prepare<<<256, 256, 0, s>>>(sp, g);
    if (n_atoms > 0) k_na_spread<<<(n_atoms + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float4*>(d_xyzq), n_atoms, sp, g);
    k_na_fft_x_fwd<<<(ky * kz + FFT_XLINES - 1) / FFT_XLINES, 256, sx, s>>>(sp, g);
    k_na_fft_y<<<ntx * kz, 256, sy, s>>>(sp, g, -1.f);
    k_na_fft_z_conv<<<ntx * ky, 256, sy, s>>>(sp, g);
    k_na_fft_y<<<ntx * kz, 256, sy, s>>>(sp, g, 1.f);
    k_na_fft_x_inv<<<(ky * kz + FFT_XLINES - 1) / FFT_XLINES, 256, sx, s>>>(sp, g);
    if (n_atoms > 0) k_na_gather<<<(n_atoms + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float4*>(d_xyzq), n_atoms, sp, g, d_forces);
    k_na_finish<<<1, 1, 0, s>>>(sp, d_energy);
    return cudaGetLastError() == cudaSuccess ? LIMA_OK : LIMA_ERR_CUDA;
}
