// nonbonded.cu — short-range LJ + real-space Coulomb over cluster pairs.
//
// Replaces compoundFarneighborShortrangeInteractionsKernel and
// compoundImmediateneighborAndSelfShortrangeInteractionsKernel
// (code/LIMA_ENGINE/src/EngineKernels.cuh:47-317) and the per-pair arithmetic of
// LJ::calcLJForceOptim (code/LIMA_ENGINE/src/LennardJonesInteractions.cuh:74-108)
// and PhysicsUtilsDevice::CalcCoulumbForce_optim / CalcCoulumbPotential_optim
// (code/LIMA_ENGINE/src/DeviceAlgorithmsPrivate.cuh:38-95):
//   F_i = [24 eps s (1-2s)/r^2 - k_e q_i q_j/r^3 (erfc(kr) + 2k/sqrt(pi) r e^{-k^2r^2})] (r_j - r_i)
//   E   = 4 eps s (s-1) + k_e q_i q_j erfc(kr)/r,   s = (sigma/r)^6
// Every unordered pair is evaluated once (Newton's third law), where the
// reference evaluates each directed pair.
//
// Work mapping (see k_nonbonded): one warp per i-cluster; each lane owns one
// j-atom of four list entries at a time and walks the 8 i-atoms.  Forces are
// added as int64 fixed point, so the result does not depend on the order in
// which warps finish.
#include "engine.h"

namespace lima {

// erfc(x) ~ t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2), t = 1/(1 + p x):
// Abramowitz & Stegun, Handbook of Mathematical Functions, 7.1.26 (|error| <=
// 1.5e-7).  Its exp(-x^2) factor is the one the Ewald force's Gaussian term
// needs, so the pair costs one exponential and one reciprocal.
constexpr float AS_P = 0.3275911f;
constexpr float AS_A1 = 0.254829592f, AS_A2 = -0.284496736f, AS_A3 = 1.421413741f;
constexpr float AS_A4 = -1.453152027f, AS_A5 = 1.061405429f;

struct PairAcc {
    double e_lj, e_c, vir;
};

// One atom pair: i-atom (xi, lji, qi) and the lane's j-atom (xj, ljj).  Returns the
// scalar fs with F_i = fs * (r_j - r_i); 0 outside the cutoff.
template <int ES, bool ENERGY>
__device__ __forceinline__ float pair_scalar(const NbParams& p, float r2, float2 lji, float2 ljj, float qq,
                                             PairAcc& acc, float& epair) {
    const float rinv = rsqrtf(r2);
    const float rinv2 = rinv * rinv;
    const float sig = lji.x + ljj.x;
    const float eps = lji.y * ljj.y;
    float s6 = sig * sig * rinv2;
    s6 = s6 * s6 * s6;
    float fs = 24.f * eps * s6 * rinv2 * (1.f - 2.f * s6);
    if (ENERGY) {
        epair = 4.f * eps * s6 * (s6 - 1.f);
        acc.e_lj += (double)epair;
    }
    if (ES != 0) {
        float fc, ec;
        if (ES == 2) {
            const float r = r2 * rinv;
            const float x = p.kappa * r;
            const float t = __fdividef(1.f, fmaf(AS_P, x, 1.f));
            const float poly = t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, AS_A5, AS_A4), AS_A3), AS_A2), AS_A1);
            const float ex = __expf(-x * x);
            const float erfc_x = poly * ex;
            fc = qq * rinv2 * rinv * fmaf(p.two_kappa_sqrtpi * r, ex, erfc_x);
            ec = qq * rinv * erfc_x;
        } else {
            fc = qq * rinv2 * rinv;
            ec = qq * rinv;
        }
        fs -= fc;
        if (ENERGY) {
            acc.e_c += (double)ec;
            epair += ec;
        }
    }
    if (p.em) fs = fmaxf(fminf(fs, 1e20f), -1e20f);
    if (ENERGY) acc.vir += 0.5 * (double)(fs * r2);  // -1/2 r_ij . f_ij
    return fs;
}

// Work mapping: one warp per i-cluster; the warp takes its list four entries at
// a time and each lane owns one j-atom (entry k0 + lane/8, j-atom lane%8).  A
// lane walks the 8 i-atoms (read from shared memory as broadcasts), keeps its
// j-atom's force in registers and adds it once per entry; the i-forces live in
// 24 registers per lane and are reduced across the warp once, after the list.
template <int ES, bool ENERGY>
__global__ void __launch_bounds__(256) k_nonbonded(DevState st, NbParams p) {
    __shared__ float4 s_xi[8][CLUSTER];
    __shared__ float2 s_lj[8][CLUSTER];
    const int wib = threadIdx.x >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= st.n_clusters) return;
    const int ci = warp;
    const int n = st.pl_count[ci];
    if (n == 0) return;
    const int sysi = st.cluster_sys[ci];
    const float Lx = st.sys[sysi].boxf[0], Ly = st.sys[sysi].boxf[1], Lz = st.sys[sysi].boxf[2];
    if (lane < CLUSTER) {
        float4 x = st.xyzq[ci * CLUSTER + lane];
        x.w *= p.ke;  // i-charges carry the Coulomb constant
        s_xi[wib][lane] = x;
        s_lj[wib][lane] = st.ljp[ci * CLUSTER + lane];
    }
    __syncwarp();
    float fi[CLUSTER][3];
    float ei[CLUSTER];     // energy steps: half of each pair energy per i-atom
#pragma unroll
    for (int a = 0; a < CLUSTER; ++a) fi[a][0] = fi[a][1] = fi[a][2] = ei[a] = 0.f;
    PairAcc acc{0.0, 0.0, 0.0};
    const int jj = lane & 7;
    const size_t base = (size_t)ci * st.pl_cap;
    for (int k0 = 0; k0 < n; k0 += 4) {
        const int k = k0 + (lane >> 3);
        unsigned bits = 0u;
        int sj = 0;
        float4 xj = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 ljj = make_float2(0.f, 0.f);
        if (k < n) {
            const int ent = st.pl_j[base + k];
            const unsigned long long mask = st.pl_mask[base + k];
            bits = (unsigned)(mask >> (8 * jj)) & 0xffu;   // bit ii: pair (ii, jj)
            const int cj = ent & ((1 << JCLUSTER_BITS) - 1);
            const int3 sh = decode_shift((unsigned)ent >> JCLUSTER_BITS);
            sj = cj * CLUSTER + jj;
            xj = st.xyzq[sj];
            ljj = st.ljp[sj];
            xj.x += sh.x * Lx;
            xj.y += sh.y * Ly;
            xj.z += sh.z * Lz;
        }
        float fjx = 0.f, fjy = 0.f, fjz = 0.f, ej = 0.f;
#pragma unroll
        for (int ii = 0; ii < CLUSTER; ++ii) {
            if ((bits >> ii) & 1u) {
                const float4 xi = s_xi[wib][ii];
                const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 <= p.rc2) {
                    float epair = 0.f;
                    const float fs = pair_scalar<ES, ENERGY>(p, r2, s_lj[wib][ii], ljj, xi.w * xj.w, acc, epair);
                    if (ENERGY) {
                        ei[ii] += 0.5f * epair;
                        ej += 0.5f * epair;
                    }
                    const float fx = fs * dx, fy = fs * dy, fz = fs * dz;
                    fi[ii][0] += fx;
                    fi[ii][1] += fy;
                    fi[ii][2] += fz;
                    fjx -= fx;
                    fjy -= fy;
                    fjz -= fz;
                }
            }
        }
        if (bits) {
            atomic_add_fixed(st.fx + sj, to_fixed(fjx, FORCE_SCALE));
            atomic_add_fixed(st.fy + sj, to_fixed(fjy, FORCE_SCALE));
            atomic_add_fixed(st.fz + sj, to_fixed(fjz, FORCE_SCALE));
            if (ENERGY) add_atom_energy(st.epot, sj, (double)ej);
        }
    }
    // i-forces: sum each of the 24 values over the warp; lane a (< 8) adds atom a's
#pragma unroll
    for (int a = 0; a < CLUSTER; ++a) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float v = fi[a][c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            fi[a][c] = v;
        }
    }
    if (ENERGY) {
#pragma unroll
        for (int a = 0; a < CLUSTER; ++a) {
            float v = ei[a];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            ei[a] = v;
        }
    }
    if (lane < CLUSTER) {
        float vx = 0.f, vy = 0.f, vz = 0.f, ve = 0.f;
#pragma unroll
        for (int a = 0; a < CLUSTER; ++a)
            if (a == lane) vx = fi[a][0], vy = fi[a][1], vz = fi[a][2], ve = ei[a];
        const int si = ci * CLUSTER + lane;
        atomic_add_fixed(st.fx + si, to_fixed(vx, FORCE_SCALE));
        atomic_add_fixed(st.fy + si, to_fixed(vy, FORCE_SCALE));
        atomic_add_fixed(st.fz + si, to_fixed(vz, FORCE_SCALE));
        if (ENERGY) add_atom_energy(st.epot, si, (double)ve);
    }
    if (ENERGY) {
        add_energy_fixed(st.energy, sysi, acc.e_lj, E_LJ);
        add_energy_fixed(st.energy, sysi, acc.e_c, E_COUL);
        add_energy_fixed(st.energy, sysi, acc.vir, E_VIRIAL);
    }
}

int launch_nonbonded(const DevState& st, const NbParams& p, bool energy, cudaStream_t s) {
    const long long threads = (long long)st.n_clusters * 32;
    const dim3 grid((unsigned)((threads + 255) / 256));
#define NB_LAUNCH(ES)                                                       \
    if (energy) k_nonbonded<ES, true><<<grid, 256, 0, s>>>(st, p);          \
    else k_nonbonded<ES, false><<<grid, 256, 0, s>>>(st, p);
    if (p.es_mode == 0) {
        NB_LAUNCH(0)
    } else if (p.es_mode == 1) {
        NB_LAUNCH(1)
    } else {
        NB_LAUNCH(2)
    }
#undef NB_LAUNCH
    return 1;
}

// Reciprocal-space exclusion correction for excluded charged pairs:
// E = -k_e q_i q_j erf(kappa r)/r.  The reference applies none (PME.cuh has no
// such term); this is the accurate-mode complement of the PME sum.
template <bool ENERGY>
__global__ void k_exclusion_correction(DevState st, BondedTerms bt, NbParams p) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    int sysi = -1;
    if (t < bt.nx) {
        const int2 pr = bt.xidx[t];
        const int si = st.slot_of[pr.x], sj = st.slot_of[pr.y];
        sysi = st.atom_sys[pr.x];
        const SysDesc& sd = st.sys[sysi];
        double d[3] = {st.px[si] - st.px[sj], st.py[si] - st.py[sj], st.pz[si] - st.pz[sj]};
        for (int k = 0; k < 3; ++k) d[k] -= sd.box[k] * rint(d[k] / sd.box[k]);
        const float dx = (float)d[0], dy = (float)d[1], dz = (float)d[2];
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float rinv = rsqrtf(r2);
        const float r = r2 * rinv;
        const float kr = p.kappa * r;
        const float qq = p.ke * st.xyzq[si].w * st.xyzq[sj].w;
        const float erf_kr = erff(kr);
        // E = -qq erf(kr)/r ; F_i = -dE/dr * (r_i - r_j)/r
        const float dEdr = -qq * (p.two_kappa_sqrtpi * __expf(-kr * kr) * rinv - erf_kr * rinv * rinv);
        const float fs = -dEdr * rinv;
        const float fx = fs * dx, fy = fs * dy, fz = fs * dz;
        atomic_add_fixed(st.fx + si, to_fixed(fx, FORCE_SCALE));
        atomic_add_fixed(st.fy + si, to_fixed(fy, FORCE_SCALE));
        atomic_add_fixed(st.fz + si, to_fixed(fz, FORCE_SCALE));
        atomic_add_fixed(st.fx + sj, to_fixed(-fx, FORCE_SCALE));
        atomic_add_fixed(st.fy + sj, to_fixed(-fy, FORCE_SCALE));
        atomic_add_fixed(st.fz + sj, to_fixed(-fz, FORCE_SCALE));
        if (ENERGY) {
            e = -(double)qq * (double)erf_kr * (double)rinv;
            add_atom_energy(st.epot, si, 0.5 * e);
            add_atom_energy(st.epot, sj, 0.5 * e);
        }
    }
    if (ENERGY) add_energy_fixed(st.energy, sysi, e, E_EXCL);
}

int launch_exclusion_correction(const DevState& st, const BondedTerms& bt, const NbParams& p,
                                bool energy, cudaStream_t s) {
    if (bt.nx == 0) return 0;
    const int TB = 256;
    if (energy)
        k_exclusion_correction<true><<<(bt.nx + TB - 1) / TB, TB, 0, s>>>(st, bt, p);
    else
        k_exclusion_correction<false><<<(bt.nx + TB - 1) / TB, TB, 0, s>>>(st, bt, p);
    return 1;
}

// Writes every (orig_i, orig_j) pair the pair kernel evaluates (mask bit set and
// r^2 <= rc^2) with i < j; order is not defined (the host sorts).
__global__ void k_pairlist_dump(DevState st, NbParams p, long long cap, int* out,
                                unsigned long long* count) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= st.n_clusters) return;
    const int ci = warp;
    const int n = st.pl_count[ci];
    const int sysi = st.cluster_sys[ci];
    const float Lx = st.sys[sysi].boxf[0], Ly = st.sys[sysi].boxf[1], Lz = st.sys[sysi].boxf[2];
    const int ii = lane & 7, jj0 = lane >> 3;
    const float4 xi = st.xyzq[ci * CLUSTER + ii];
    const int ai = st.orig[ci * CLUSTER + ii];
    const size_t base = (size_t)ci * st.pl_cap;
    for (int k = 0; k < n; ++k) {
        const int ent = st.pl_j[base + k];
        const unsigned long long mask = st.pl_mask[base + k];
        const int cj = ent & ((1 << JCLUSTER_BITS) - 1);
        const int3 sh = decode_shift((unsigned)ent >> JCLUSTER_BITS);
        for (int h = 0; h < 2; ++h) {
            const int jj = jj0 + 4 * h;
            const float4 xj = st.xyzq[cj * CLUSTER + jj];
            const float dx = xj.x + sh.x * Lx - xi.x;
            const float dy = xj.y + sh.y * Ly - xi.y;
            const float dz = xj.z + sh.z * Lz - xi.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (((mask >> (jj * 8 + ii)) & 1ull) && r2 <= p.rc2) {
                const int aj = st.orig[cj * CLUSTER + jj];
                const unsigned long long w = atomicAdd(count, 1ull);
                if ((long long)w < cap) {
                    out[2 * w] = min(ai, aj);
                    out[2 * w + 1] = max(ai, aj);
                }
            }
        }
    }
}

int launch_pairlist_dump(const DevState& st, const NbParams& p, long long cap, int* out_pairs,
                         unsigned long long* out_count, cudaStream_t s) {
    const long long threads = (long long)st.n_clusters * 32;
    k_pairlist_dump<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(st, p, cap, out_pairs, out_count);
    return 1;
}

}  // namespace lima
