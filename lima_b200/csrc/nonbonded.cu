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
// row of the list (a j-atom with an 8-bit mask of the i-atoms it meets) and
// walks the 8 i-atoms.  Forces are added as int64 fixed point, so the result
// does not depend on the order in which warps finish.
#include <type_traits>

#include "engine.h"
#include "packed.cuh"

namespace lima {

// erfc(x) ~ t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2), t = 1/(1 + p x):
// Abramowitz & Stegun, Handbook of Mathematical Functions, 7.1.26 (|error| <=
// 1.5e-7).  Its exp(-x^2) factor is the one the Ewald force's Gaussian term
// needs, so the pair costs one exponential and one reciprocal.
// (AS_P, the p of the form, is in engine.h: the host folds it into NbParams::p_kappa)
constexpr float AS_A1 = 0.254829592f, AS_A2 = -0.284496736f, AS_A3 = 1.421413741f;
constexpr float AS_A4 = -1.453152027f, AS_A5 = 1.061405429f;

// Energy minimisation: every LJ pair force passes through the reference's tanh
// activation, |F| -> A tanh(|F| / A) with A = 1e8 in its 1/24 J/mol/nm force unit
// (LennardJonesInteractions.cuh:85-101 with EngineUtils.cuh:112-140), after its
// +-1e20 guard on the scalar.  fsl multiplies the pair vector, r is the distance.
__device__ __forceinline__ float em_lj_clamp(float fsl, float r) {
    constexpr float A = 24.f * 1e8f;   // [J/mol/nm]
    fsl = fmaxf(fminf(fsl, 24.f * 1e20f), -24.f * 1e20f);
    const float f = fabsf(fsl) * r;
    return fsl * (A * tanhf(f / A) / (f + 24.f * 1e-8f));
}

// 2^x, the hardware approximation (PTX ex2.approx.ftz.f32)
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// erfc for the energy of energy steps: erfc(x) = t (c0 + c1 t + ... + c7 t^7) e^{-x^2}
// with the force's t = 1/(1 + p x) and e^{-x^2}, so an energy step adds only this
// polynomial to the force's arithmetic.  The coefficients are this build's own
// weighted least-squares fit of erfc(x) e^{x^2} over x in [0, 5.5]
// (lima_b200/csrc/erfcx_fit.py): relative error below 6e-8 in exact arithmetic,
// 4.4e-7 evaluated in FP32 — the relative bound a total energy needs, where the
// force's A&S form only bounds the absolute error (1.5e-7).  Past x = 5.5, where
// erfc < 1e-14, the polynomial is extrapolated (2e-4 relative up to x = 30).
constexpr float EC0 = 0.185084581f, EC1 = 0.180205658f, EC2 = 0.209264949f, EC3 = 0.014182996f;
constexpr float EC4 = 0.474507362f, EC5 = -0.428924263f, EC6 = 0.509979844f, EC7 = -0.144301191f;

// erfc(x) from the force's t and e^{-x^2} (packed pairs)
__device__ __forceinline__ f2p erfc_from_t(f2p t, f2p ex) {
    f2p q = fma2(t, splat2(EC7), splat2(EC6));
    q = fma2(q, t, splat2(EC5));
    q = fma2(q, t, splat2(EC4));
    q = fma2(q, t, splat2(EC3));
    q = fma2(q, t, splat2(EC2));
    q = fma2(q, t, splat2(EC1));
    q = fma2(q, t, splat2(EC0));
    return mul2(mul2(q, t), ex);
}

// 1/sqrt(x) and 1/x, the hardware approximations with subnormal inputs and
// results flushed to zero: the pair kernel's r^2 (>= 1e-4 nm^2 for any pair
// that is kept) and 1 + p kappa r are never subnormal, and the flush spares the
// subnormal fix-up instructions of the non-flushing forms in the inner loop
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One pair-list row: the lane's j-atom against the 8 i-atoms of its warp's
// cluster, two at a time, (2 ip, 2 ip + 1) for ip = 0..3, in packed FP32.
// sxy, szq, slj: the cluster's i-atom pairs in shared memory, (x0, x1, y0, y1),
// (z0, z1, -q0 ke, -q1 ke), (sigma0/2, sigma1/2, 24 sqrt(eps0), 24 sqrt(eps1)).
// NLJ: the i-pairs ip < NLJ carry LJ; the pairs above hold only atoms with
// eps = 0, whose LJ force and energy are exactly zero against any j-atom, so
// their LJ arithmetic is left out (a cluster's atoms with LJ come first in its
// slots; in water 60 % of the i-pairs are LJ-free).  Leaving it out changes no
// bit: the LJ term would add +-0 to the same Coulomb product.
// The pair force is rinv^2 (LJ + Coulomb) with both terms taken times r^2:
//   LJ r^2 = 24 eps s6 (1 - 2 s6),  Coulomb r^2 = -qn e^{-k^2 r^2} (poly/r + 2k/sqrt(pi))
// (Ewald), -qn/r (plain cutoff).  Every lane evaluates both elements of every
// pair (straight-line code over the four pairs, which the scheduler
// interleaves); the mask bit of each element is folded into its cutoff (rc^2,
// or -1: never met) and elements outside the mask or the cutoff — possibly
// non-finite, e.g. a padding slot at distance 0 — are dropped by the select.
template <int ES, int EN, bool EM, int NLJ>
__device__ __forceinline__ void pair_row(const float4* sxy, const float4* szq, const float4* slj,
                                         const NbParams& p, unsigned bits, float4 xj, float2 ljj,
                                         f2p (&fix)[4], f2p (&fiy)[4], f2p (&fiz)[4], f2p (&ei)[4],
                                         f2p& fjx, f2p& fjy, f2p& fjz, f2p& ej,
                                         f2p& r_elj, f2p& r_ec, f2p& r_vir) {
    constexpr bool ENERGY = EN > 0, ATOM = EN > 1;
    const f2p zero2 = splat2(0.f), one2 = splat2(1.f), mtwo2 = splat2(-2.f);
    const f2p jx = splat2(xj.x), jy = splat2(xj.y), jz = splat2(xj.z);
    const f2p jsig = splat2(ljj.x), jeps = splat2(ljj.y), jq = splat2(xj.w);
#pragma unroll
    for (int ip = 0; ip < 4; ++ip) {
        const bool lj = ip < NLJ;
        const float tha = (bits >> (2 * ip)) & 1u ? p.rc2 : -1.f;
        const float thb = (bits >> (2 * ip + 1)) & 1u ? p.rc2 : -1.f;
        const float4 vxy = sxy[ip], vzq = szq[ip];
        const f2p dx = sub2(jx, pk2(vxy.x, vxy.y));
        const f2p dy = sub2(jy, pk2(vxy.z, vxy.w));
        const f2p dz = sub2(jz, pk2(vzq.x, vzq.y));
        const f2p r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
        const float2 r2v = up2(r2);
        const bool oka = r2v.x <= tha, okb = r2v.y <= thb;
        const f2p rinv = pk2(rsqrt_ftz(r2v.x), rsqrt_ftz(r2v.y));
        const f2p rinv2 = mul2(rinv, rinv);
        f2p eps24 = zero2, s6 = zero2, lj_r2 = zero2, flj = zero2;
        if (lj) {
            const float4 vlj = slj[ip];
            const f2p sig = add2(pk2(vlj.x, vlj.y), jsig);
            eps24 = mul2(pk2(vlj.z, vlj.w), jeps);
            const f2p s2 = mul2(mul2(sig, sig), rinv2);
            s6 = mul2(mul2(s2, s2), s2);
            lj_r2 = mul2(mul2(eps24, s6), fma2(s6, mtwo2, one2));   // 24 eps s6 (1 - 2 s6)
            if (EM) {
                // energy minimisation: the LJ force alone passes the reference's clamp
                const float2 v = up2(mul2(lj_r2, rinv2)), rr = up2(mul2(r2, rinv));
                flj = pk2(em_lj_clamp(v.x, rr.x), em_lj_clamp(v.y, rr.y));
            }
        }
        f2p fs = zero2, ec = zero2;
        if (ES != 0) {
            // qn = -k_e q_i q_j (the sign rides on the i-charge)
            const f2p qn = mul2(pk2(vzq.z, vzq.w), jq);
            if (ES == 2) {
                const f2p r = mul2(r2, rinv);
                const float2 den = up2(fma2(splat2(p.p_kappa), r, one2));   // 1 + p kappa r
                const f2p t = pk2(rcp_ftz(den.x), rcp_ftz(den.y));
                // erfc(kappa r) = poly e^{-kappa^2 r^2}
                const f2p poly = mul2(t, fma2(t, fma2(t, fma2(t, fma2(t, splat2(AS_A5), splat2(AS_A4)),
                                                            splat2(AS_A3)), splat2(AS_A2)), splat2(AS_A1)));
                const float2 xs = up2(mul2(r2, splat2(p.mk2_log2e)));
                const f2p ex = pk2(ex2_approx(xs.x), ex2_approx(xs.y));
                const f2p g = fma2(poly, rinv, splat2(p.two_kappa_sqrtpi));
                const f2p qe = mul2(qn, ex);
                if (EM) fs = lj ? fma2(mul2(qe, rinv2), g, flj) : mul2(mul2(qe, rinv2), g);
                else fs = mul2(lj ? fma2(qe, g, lj_r2) : mul2(qe, g), rinv2);
                if (ENERGY) ec = mul2(mul2(qn, rinv), erfc_from_t(t, ex));   // minus the pair energy
            } else {
                if (EM) fs = lj ? fma2(mul2(qn, rinv2), rinv, flj) : mul2(mul2(qn, rinv2), rinv);
                else fs = mul2(lj ? fma2(qn, rinv, lj_r2) : mul2(qn, rinv), rinv2);
                if (ENERGY) ec = mul2(qn, rinv);   // minus the pair energy
            }
        } else if (lj) {
            fs = EM ? flj : mul2(lj_r2, rinv2);
        }
        float2 fsv = up2(fs);
        if (EM) {   // a non-finite Coulomb term (coincident atoms) kept finite
            fsv.x = fmaxf(fminf(fsv.x, 1e20f), -1e20f);
            fsv.y = fmaxf(fminf(fsv.y, 1e20f), -1e20f);
        }
        fs = pk2(oka ? fsv.x : 0.f, okb ? fsv.y : 0.f);
        // force on i: fs d; on j: -fs d (both summed as +fs d, j negated at the end)
        fix[ip] = fma2(fs, dx, fix[ip]);
        fiy[ip] = fma2(fs, dy, fiy[ip]);
        fiz[ip] = fma2(fs, dz, fiz[ip]);
        fjx = fma2(fs, dx, fjx);
        fjy = fma2(fs, dy, fjy);
        fjz = fma2(fs, dz, fjz);
        if (ENERGY) {
            // the row sums carry minus the Coulomb energy and six times the LJ energy
            // (24 eps s6 (s6 - 1) = 6 x 4 eps s6 (s6 - 1)); the kernel's FP64 totals
            // take the sign and the sixth once per warp.  Dropped like the force.
            const float2 ecv = up2(ec);
            const f2p ecm = pk2(oka ? ecv.x : 0.f, okb ? ecv.y : 0.f);
            f2p elj6 = zero2;
            if (lj) {
                const float2 eljv = up2(mul2(eps24, mul2(s6, sub2(s6, one2))));
                elj6 = pk2(oka ? eljv.x : 0.f, okb ? eljv.y : 0.f);
                r_elj = add2(r_elj, elj6);
            }
            // the row's sums in packed FP32 (at most 8 terms), then FP64 per row
            r_ec = add2(r_ec, ecm);
            r_vir = fma2(fs, r2, r_vir);   // fs is already dropped; -1/2 r_ij . f_ij = fs r^2 / 2
            if (ATOM) {   // half of each pair's energy to each atom
                const f2p eh = lj ? fma2(elj6, splat2(1.f / 12.f), mul2(ecm, splat2(-0.5f)))
                                  : mul2(ecm, splat2(-0.5f));
                ei[ip] = add2(ei[ip], eh);
                ej = add2(ej, eh);
            }
        }
    }
}

// The number of leading i-pairs (2 ip, 2 ip + 1) of a cluster that hold an atom
// with LJ (eps != 0), from the ballot of those atoms over the cluster's 8 slots.
__device__ __forceinline__ int lj_pairs_of(unsigned lj_atoms) {
    return lj_atoms ? ((31 - __clz(lj_atoms)) >> 1) + 1 : 0;
}

// Calls f(std::integral_constant<int, NLJ>) for the runtime count nlj (0..4), so
// that a warp's whole walk over its rows is one specialisation.
template <typename F>
__device__ __forceinline__ void with_lj_pairs(int nlj, F&& f) {
    switch (nlj) {
        case 0: f(std::integral_constant<int, 0>{}); break;
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 3: f(std::integral_constant<int, 3>{}); break;
        default: f(std::integral_constant<int, 4>{}); break;
    }
}

// Work mapping: one warp per i-cluster; the warp takes its list 32 rows at a
// time and each lane owns one row: a j-atom whose 8-bit mask names the i-atoms
// it interacts with (rows whose mask would be empty are not in the list, so no
// lane works on a j-atom out of range of the whole i-cluster).  A lane walks the
// 8 i-atoms two at a time, (2 ip, 2 ip + 1) for ip = 0..3, in packed FP32 (read as
// float4 pairs from shared memory), keeps its j-atom's force in a packed
// register and adds it once per row; the i-forces live in 12 packed registers
// per lane and are reduced across the warp once, after the list.  The walk is
// compiled once per count of the cluster's i-pairs with LJ (pair_row's NLJ),
// chosen per warp from a ballot of its atoms' epsilon.
// Pair arithmetic per lane and the order of every sum are fixed, so results
// are bit-reproducible.
// EN: 0 forces only, 1 forces and energy totals, 2 also per-atom energy shares.
// PF: software-pipelined loads — the row two chunks ahead and the j-atom one
// chunk ahead are loaded before the current row's arithmetic, so their latency
// overlaps it; the rows are worked in the same order, so the results are the
// same bits either way.
// EM: the energy-minimisation variant (force only, the per-pair LJ clamp above).
// SPLIT: the rows of a cluster may be split over several warps (a small
// system's engine, see below); without it a warp is a whole cluster.
template <int ES, int EN, bool PF, bool EM = false, bool SPLIT = false>
__global__ void __launch_bounds__(256, (EN || EM) ? 2 : 3) k_nonbonded(DevState st, NbParams p) {
    constexpr bool ENERGY = EN > 0, ATOM = EN > 1;
    // per warp, i-atom pairs (2 ip, 2 ip + 1): (x0, x1, y0, y1), (z0, z1, -q0 ke, -q1 ke),
    // (sigma0/2, sigma1/2, 24 sqrt(eps0), 24 sqrt(eps1))
    __shared__ float4 s_xy[8][4], s_zq[8][4], s_lj[8][4];
    const int wib = threadIdx.x >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    // warp -> (system, i-cluster, part): a small system's rows are split over
    // nb_parts warps (parts of 32-row multiples, so a row meets the same lane
    // either way); the system is found by binary search over the warp offsets
    if (warp >= st.nb_warps) return;
    int sysi, ci, parts = 1, part = 0;
    if (!SPLIT) {   // one warp per cluster: no lookups before the row loads
        ci = warp;
        sysi = st.cluster_sys[ci];
    } else {
        sysi = 0;
        for (int hi = st.n_sys - 1; sysi < hi;) {
            const int mid = (sysi + hi + 1) >> 1;
            if (st.nb_warp_off[mid] <= warp) sysi = mid;
            else hi = mid - 1;
        }
        parts = max(1, st.sys[sysi].nb_parts);
        const int local = warp - st.nb_warp_off[sysi], lp = __ffs(parts) - 1;
        ci = st.sys[sysi].cluster_cap_off + (local >> lp);
        part = local & (parts - 1);
    }
    const int n_rows = min(st.walk_count[ci], st.pl_cap);
    const int chunk = SPLIT ? ((n_rows + parts - 1) / parts + 31) & ~31 : n_rows;
    const int k_begin = SPLIT ? part * chunk : 0;
    const int n = SPLIT ? min(n_rows, k_begin + chunk) : n_rows;   // end of this warp's rows
    if (k_begin >= n) return;
    const float Lx = st.sys[sysi].boxf[0], Ly = st.sys[sysi].boxf[1], Lz = st.sys[sysi].boxf[2];
    float2 lj_i = make_float2(0.f, 0.f);
    if (lane < CLUSTER) {
        const float4 x = st.xyzq[ci * CLUSTER + lane];
        lj_i = st.ljp[ci * CLUSTER + lane];
        const int ip = lane >> 1, h = lane & 1;   // pair ip holds atoms 2 ip and 2 ip + 1
        float* xy = reinterpret_cast<float*>(&s_xy[wib][ip]);
        float* zq = reinterpret_cast<float*>(&s_zq[wib][ip]);
        float* lv = reinterpret_cast<float*>(&s_lj[wib][ip]);
        xy[h] = x.x;
        xy[2 + h] = x.y;
        zq[h] = x.z;
        zq[2 + h] = -x.w * p.ke;  // i-charges carry minus the Coulomb constant
        lv[h] = lj_i.x;
        lv[2 + h] = 24.f * lj_i.y;  // the LJ force prefactor folded into the i side
    }
    // i-pairs with LJ: the cluster's atoms with eps != 0 lead its slots
    const int nlj = lj_pairs_of(__ballot_sync(0xffffffffu, lj_i.y != 0.f));
    __syncwarp();
    f2p fix[4], fiy[4], fiz[4], ei[4];
    const f2p zero2 = splat2(0.f);
#pragma unroll
    for (int ip = 0; ip < 4; ++ip) fix[ip] = fiy[ip] = fiz[ip] = ei[ip] = zero2;
    // energy steps: per-lane FP64 sums of the pair energies and virial terms
    double s_elj = 0.0, s_ec = 0.0, s_vir = 0.0;
    const size_t base = (size_t)ci * st.pl_cap;
    // one row: its mask, j slot, j position with the row's image applied, j LJ
    auto load_j = [&](int k, int2 row, unsigned& bits, int& sj, float4& xj, float2& ljj) {
        bits = 0u;
        sj = 0;
        xj = make_float4(0.f, 0.f, 0.f, 0.f);
        ljj = make_float2(0.f, 0.f);
        if (k < n) {
            bits = (unsigned)row.y & 0xffu;   // bit ii: pair (ii, this j-atom)
            const unsigned img = (unsigned)row.y >> ROW_SHIFT_BIT;
            sj = row.x;
            xj = st.xyzq[sj];
            ljj = st.ljp[sj];
            // image shift s L with s + 1 in two bits per axis
            xj.x += fmaf((float)(img & 3u), Lx, -Lx);
            xj.y += fmaf((float)((img >> 2) & 3u), Ly, -Ly);
            xj.z += fmaf((float)(img >> 4), Lz, -Lz);
        }
    };
    auto load_rowid = [&](int k) { return k < n ? st.walk_row[base + k] : make_int2(0, 0); };
    auto load_row = [&](int k, unsigned& bits, int& sj, float4& xj, float2& ljj) {
        load_j(k, load_rowid(k), bits, sj, xj, ljj);
    };
    // the warp's rows, one specialisation per number of LJ i-pairs
    auto walk = [&](auto nlj_c) {
        constexpr int NLJ = decltype(nlj_c)::value;
        auto do_row = [&](unsigned bits, int sj, float4 xj, float2 ljj) {
            f2p fjx = zero2, fjy = zero2, fjz = zero2, ej = zero2;
            f2p r_elj = zero2, r_ec = zero2, r_vir = zero2;   // the row's energy sums (energy steps)
            pair_row<ES, EN, EM, NLJ>(s_xy[wib], s_zq[wib], s_lj[wib], p, bits, xj, ljj, fix, fiy, fiz, ei,
                                      fjx, fjy, fjz, ej, r_elj, r_ec, r_vir);
            if (ENERGY) {
                const float2 a = up2(r_elj), c = up2(r_ec), v = up2(r_vir);
                s_elj += (double)a.x + (double)a.y;
                s_ec -= (double)c.x + (double)c.y;
                s_vir += (double)v.x + (double)v.y;
            }
            if (bits) {
                const float2 x = up2(fjx), y = up2(fjy), z = up2(fjz);
                atomic_add_fixed(st.fx + sj, to_fixed(-(x.x + x.y), FORCE_SCALE));
                atomic_add_fixed(st.fy + sj, to_fixed(-(y.x + y.y), FORCE_SCALE));
                atomic_add_fixed(st.fz + sj, to_fixed(-(z.x + z.y), FORCE_SCALE));
                if (ATOM) {
                    const float2 e = up2(ej);
                    add_atom_energy(st.epot, sj, (double)(e.x + e.y));
                }
            }
        };
        if (PF) {
            // software pipeline: while a lane works on row k, the j-atom loads of row
            // k + 32 and the row load of row k + 64 are in flight
            unsigned ba;
            int sa;
            float4 xa;
            float2 la;
            int2 rb = load_rowid(k_begin + 32 + lane);
            load_row(k_begin + lane, ba, sa, xa, la);
            for (int k0 = k_begin; k0 < n; k0 += 32) {
                const int2 rc = load_rowid(k0 + 64 + lane);
                unsigned bb;
                int sb;
                float4 xb;
                float2 lb;
                load_j(k0 + 32 + lane, rb, bb, sb, xb, lb);
                do_row(ba, sa, xa, la);
                ba = bb, sa = sb, xa = xb, la = lb, rb = rc;
            }
        } else {
            for (int k0 = k_begin; k0 < n; k0 += 32) {
                unsigned ba;
                int sa;
                float4 xa;
                float2 la;
                load_row(k0 + lane, ba, sa, xa, la);
                do_row(ba, sa, xa, la);
            }
        }
    };
    with_lj_pairs(nlj, walk);
    // i-forces: sum each of the 24 values over the warp; lane a (< 8) adds atom a's
    float fi[CLUSTER][3], eiv[CLUSTER];
#pragma unroll
    for (int ip = 0; ip < 4; ++ip) {
        const float2 x = up2(fix[ip]), y = up2(fiy[ip]), z = up2(fiz[ip]), e = up2(ei[ip]);
        fi[2 * ip][0] = x.x, fi[2 * ip][1] = y.x, fi[2 * ip][2] = z.x, eiv[2 * ip] = e.x;
        fi[2 * ip + 1][0] = x.y, fi[2 * ip + 1][1] = y.y, fi[2 * ip + 1][2] = z.y, eiv[2 * ip + 1] = e.y;
    }
#pragma unroll
    for (int a = 0; a < CLUSTER; ++a) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float v = fi[a][c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            fi[a][c] = v;
        }
        if (ATOM) {
            float v = eiv[a];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            eiv[a] = v;
        }
    }
    if (lane < CLUSTER) {
        float vx = 0.f, vy = 0.f, vz = 0.f, ve = 0.f;
#pragma unroll
        for (int a = 0; a < CLUSTER; ++a)
            if (a == lane) vx = fi[a][0], vy = fi[a][1], vz = fi[a][2], ve = eiv[a];
        const int si = ci * CLUSTER + lane;
        atomic_add_fixed(st.fx + si, to_fixed(vx, FORCE_SCALE));
        atomic_add_fixed(st.fy + si, to_fixed(vy, FORCE_SCALE));
        atomic_add_fixed(st.fz + si, to_fixed(vz, FORCE_SCALE));
        if (ATOM) add_atom_energy(st.epot, si, (double)ve);
    }
    if (ENERGY) {
        add_energy_fixed(st.energy, sysi, s_elj * (1.0 / 6.0), E_LJ);
        add_energy_fixed(st.energy, sysi, s_ec, E_COUL);
        add_energy_fixed(st.energy, sysi, 0.5 * s_vir, E_VIRIAL);
    }
}

// ------------------------------------------------------- staged pair kernel
// cp.async (sm_80+ LDGSTS): copies from global to shared memory that complete
// asynchronously; wait_all makes the calling thread's copies visible to it.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Per warp: three stages of 32 pair-list rows and of their j-atoms' (x, y, z, q)
// and LJ parameters, plus the i-cluster's packed atom pairs.
constexpr int NB_STAGES = 3;
struct alignas(16) NbWarpStage {
    float4 xj[NB_STAGES][32];
    float2 lj[NB_STAGES][32];
    int2 row[NB_STAGES][32];
    float4 xy[4], zq[4], ljp[4];
};

// The pair kernel with its list rows and j-atoms staged through shared memory.
// The same pair arithmetic and per-lane work as k_nonbonded (one lane per list
// row, the 8 i-atoms in packed pairs (2 ip, 2 ip + 1)); what changes is how the
// operands arrive and how clusters reach warps:
//  * staging: while a warp works on chunk c of its cluster's list (32 rows),
//    the j-atoms of chunk c + 1 and the rows of chunk c + 2 are already in
//    flight as cp.async copies into the warp's shared-memory stages, so the
//    dependent row -> j-atom loads never stall the arithmetic (each lane
//    copies its own row and that row's j-atom, three stages deep);
//  * persistence: a grid of a few CTAs per SM whose warps take i-clusters from
//    a counter (atomicAdd) until the list is done, so no partial last wave;
//  * both the i-force and the j-force sums take fs * d with one FMA each.
// Every sum is still rounded to int64 fixed point before it is added, so the
// results do not depend on which warp takes which cluster.
template <int ES, int EN, bool EM>
__global__ void __launch_bounds__(256, (EN || EM) ? 2 : 3) k_nonbonded_staged(DevState st, NbParams p, int* counter) {
    constexpr bool ENERGY = EN > 0, ATOM = EN > 1;
    extern __shared__ __align__(16) unsigned char nb_smem[];
    NbWarpStage& S = reinterpret_cast<NbWarpStage*>(nb_smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const f2p zero2 = splat2(0.f);
    for (;;) {
        int ci = 0;
        if (lane == 0) ci = atomicAdd(counter, 1);
        ci = __shfl_sync(0xffffffffu, ci, 0);
        if (ci >= st.n_clusters) break;
        const int n = min(st.walk_count[ci], st.pl_cap);
        if (n == 0) continue;
        const int sysi = st.cluster_sys[ci];
        const float Lx = st.sys[sysi].boxf[0], Ly = st.sys[sysi].boxf[1], Lz = st.sys[sysi].boxf[2];
        const size_t base = (size_t)ci * st.pl_cap;
        const int nchunk = (n + 31) >> 5;
        // rows of chunk 0 first: the j-atom copies need them
        if (lane < n) cp_async8(&S.row[0][lane], &st.walk_row[base + lane]);
        cp_async_commit();
        if (lane < CLUSTER) {
            const float4 x = st.xyzq[ci * CLUSTER + lane];
            const float2 lj = st.ljp[ci * CLUSTER + lane];
            const int ip = lane >> 1, h = lane & 1;   // pair ip holds atoms 2 ip and 2 ip + 1
            float* xy = reinterpret_cast<float*>(&S.xy[ip]);
            float* zq = reinterpret_cast<float*>(&S.zq[ip]);
            float* lv = reinterpret_cast<float*>(&S.ljp[ip]);
            xy[h] = x.x;
            xy[2 + h] = x.y;
            zq[h] = x.z;
            zq[2 + h] = -x.w * p.ke;  // i-charges carry minus the Coulomb constant
            lv[h] = lj.x;
            lv[2 + h] = 24.f * lj.y;  // the LJ force prefactor folded into the i side
        }
        cp_async_wait_all();
        // j-atoms of chunk 0 and rows of chunk 1
        if (lane < n) {
            const int sj = S.row[0][lane].x;
            cp_async16(&S.xj[0][lane], &st.xyzq[sj]);
            cp_async8(&S.lj[0][lane], &st.ljp[sj]);
        }
        if (32 + lane < n) cp_async8(&S.row[1][lane], &st.walk_row[base + 32 + lane]);
        cp_async_commit();
        __syncwarp();   // the i-atoms written by lanes 0-7 are visible to the warp

        f2p fix[4], fiy[4], fiz[4], ei[4];
#pragma unroll
        for (int ip = 0; ip < 4; ++ip) fix[ip] = fiy[ip] = fiz[ip] = ei[ip] = zero2;
        double s_elj = 0.0, s_ec = 0.0, s_vir = 0.0;   // energy steps: per-lane FP64 sums
        for (int c = 0; c < nchunk; ++c) {
            const int b0 = c % NB_STAGES, b1 = (c + 1) % NB_STAGES, b2 = (c + 2) % NB_STAGES;
            cp_async_wait_all();        // rows of c + 1 and j-atoms of c have landed
            const int k = (c << 5) + lane;
            const int2 row = k < n ? S.row[b0][lane] : make_int2(0, 0);
            // next: j-atoms of chunk c + 1, rows of chunk c + 2
            if (k + 32 < n) {
                const int sj1 = S.row[b1][lane].x;
                cp_async16(&S.xj[b1][lane], &st.xyzq[sj1]);
                cp_async8(&S.lj[b1][lane], &st.ljp[sj1]);
            }
            if (k + 64 < n) cp_async8(&S.row[b2][lane], &st.walk_row[base + k + 64]);
            cp_async_commit();

            const unsigned bits = (unsigned)row.y & 0xffu;   // bit ii: pair (ii, this j-atom); 0 past the list
            const unsigned img = (unsigned)row.y >> ROW_SHIFT_BIT;
            const int sj = row.x;
            // lanes past the list take zeros, never a stage slot's stale contents
            // (a non-finite stale value times fs = 0 would reach the sums)
            float4 xj = k < n ? S.xj[b0][lane] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float2 ljj = k < n ? S.lj[b0][lane] : make_float2(0.f, 0.f);
            xj.x += fmaf((float)(img & 3u), Lx, -Lx);
            xj.y += fmaf((float)((img >> 2) & 3u), Ly, -Ly);
            xj.z += fmaf((float)(img >> 4), Lz, -Lz);
            f2p fjx = zero2, fjy = zero2, fjz = zero2, ej = zero2;
            f2p r_elj = zero2, r_ec = zero2, r_vir = zero2;   // the row's energy sums (energy steps)
            // every i-pair takes the LJ arithmetic here (the same bits as leaving it
            // out for the LJ-free pairs, as the plain kernel does)
            pair_row<ES, EN, EM, 4>(S.xy, S.zq, S.ljp, p, bits, xj, ljj, fix, fiy, fiz, ei, fjx, fjy, fjz, ej,
                                    r_elj, r_ec, r_vir);
            if (ENERGY) {
                const float2 a = up2(r_elj), c = up2(r_ec), v = up2(r_vir);
                s_elj += (double)a.x + (double)a.y;
                s_ec -= (double)c.x + (double)c.y;
                s_vir += (double)v.x + (double)v.y;
            }
            if (bits) {
                const float2 x = up2(fjx), y = up2(fjy), z = up2(fjz);
                atomic_add_fixed(st.fx + sj, to_fixed(-(x.x + x.y), FORCE_SCALE));
                atomic_add_fixed(st.fy + sj, to_fixed(-(y.x + y.y), FORCE_SCALE));
                atomic_add_fixed(st.fz + sj, to_fixed(-(z.x + z.y), FORCE_SCALE));
                if (ATOM) {
                    const float2 e = up2(ej);
                    add_atom_energy(st.epot, sj, (double)(e.x + e.y));
                }
            }
        }
        // i-forces: sum each of the 24 values over the warp; lane a (< 8) adds atom a's
        float fi[CLUSTER][3], eiv[CLUSTER];
#pragma unroll
        for (int ip = 0; ip < 4; ++ip) {
            const float2 x = up2(fix[ip]), y = up2(fiy[ip]), z = up2(fiz[ip]), e = up2(ei[ip]);
            fi[2 * ip][0] = x.x, fi[2 * ip][1] = y.x, fi[2 * ip][2] = z.x, eiv[2 * ip] = e.x;
            fi[2 * ip + 1][0] = x.y, fi[2 * ip + 1][1] = y.y, fi[2 * ip + 1][2] = z.y, eiv[2 * ip + 1] = e.y;
        }
#pragma unroll
        for (int a = 0; a < CLUSTER; ++a) {
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                float v = fi[a][cc];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                fi[a][cc] = v;
            }
            if (ATOM) {
                float v = eiv[a];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                eiv[a] = v;
            }
        }
        if (lane < CLUSTER) {
            float vx = 0.f, vy = 0.f, vz = 0.f, ve = 0.f;
#pragma unroll
            for (int a = 0; a < CLUSTER; ++a)
                if (a == lane) vx = fi[a][0], vy = fi[a][1], vz = fi[a][2], ve = eiv[a];
            const int si = ci * CLUSTER + lane;
            atomic_add_fixed(st.fx + si, to_fixed(vx, FORCE_SCALE));
            atomic_add_fixed(st.fy + si, to_fixed(vy, FORCE_SCALE));
            atomic_add_fixed(st.fz + si, to_fixed(vz, FORCE_SCALE));
            if (ATOM) add_atom_energy(st.epot, si, (double)ve);
        }
        if (ENERGY) {
            add_energy_fixed(st.energy, sysi, s_elj * (1.0 / 6.0), E_LJ);
            add_energy_fixed(st.energy, sysi, s_ec, E_COUL);
            add_energy_fixed(st.energy, sysi, 0.5 * s_vir, E_VIRIAL);
        }
        cp_async_wait_all();   // nothing of this cluster still in flight into the stages
        __syncwarp();          // every lane done with the i-atoms before the next cluster's
    }
}

// Staged launch shapes (shape bit 3): bit 1 selects 128-thread blocks, bit 0
// fewer resident blocks per SM (room for the PME and bonded kernels beside
// them).  The grid is persistent: blocks per SM x SM count.
template <int ES>
static void launch_nb_staged(const DevState& st, const NbParams& p, bool energy, int shape, cudaStream_t s) {
    const int tb = (shape & 2) ? 128 : 256;
    const size_t smem = (size_t)(tb / 32) * sizeof(NbWarpStage);
    static std::atomic<unsigned long long> attr{0ull};
    once_per_device(attr, [] {
        const int mx = 8 * (int)sizeof(NbWarpStage);
        cudaFuncSetAttribute(k_nonbonded_staged<ES, 0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_nonbonded_staged<ES, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_nonbonded_staged<ES, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_nonbonded_staged<ES, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    });
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int warps_per_sm = (shape & 1) ? 16 : 24;
    const long long need = ((long long)st.n_clusters * 32 + tb - 1) / tb;
    const unsigned grid = (unsigned)std::max(1ll, std::min<long long>(need, (long long)sms * (warps_per_sm * 32 / tb)));
    cudaMemsetAsync(st.nb_counter, 0, sizeof(int), s);
    if (p.em && !energy) k_nonbonded_staged<ES, 0, true><<<grid, tb, smem, s>>>(st, p, st.nb_counter);
    else if (!energy) k_nonbonded_staged<ES, 0, false><<<grid, tb, smem, s>>>(st, p, st.nb_counter);
    else if (st.atom_energy) k_nonbonded_staged<ES, 2, false><<<grid, tb, smem, s>>>(st, p, st.nb_counter);
    else k_nonbonded_staged<ES, 1, false><<<grid, tb, smem, s>>>(st, p, st.nb_counter);
}

// Launch shapes of the force-only pair kernel (results are identical for every
// shape: the work of a warp does not depend on the block it sits in):
//   bit 0: reserve unused shared memory so that the kernel holds at most 24-28
//          warps of an SM, leaving registers, shared memory and block slots to
//          the PME and bonded kernels of the same step on their higher-priority
//          streams (helps when the PME chain is long next to the pair kernel);
//   bit 1: 128-thread blocks instead of 256;
//   bit 2: two rows' loads in flight per lane (PF).
// The engine's autotuner times the shapes on the running system.
template <int ES, bool SP>
static void launch_nb_shape(const DevState& st, const NbParams& p, bool energy, int shape, cudaStream_t s) {
    const long long threads = (long long)st.nb_warps * 32;
    if (p.em && !energy) {   // energy minimisation: forces with the per-pair LJ clamp
        k_nonbonded<ES, 0, false, true, SP><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(st, p);
        return;
    }
    const int tb = (shape & 2) ? 128 : 256;
    const dim3 grid((unsigned)((threads + tb - 1) / tb));
    if (energy) {
        if (st.atom_energy) k_nonbonded<ES, 2, false, false, SP><<<grid, tb, 0, s>>>(st, p);
        else k_nonbonded<ES, 1, false, false, SP><<<grid, tb, 0, s>>>(st, p);
        return;
    }
    // 24 to 28 warps per SM: 3 blocks of 256 threads (60 KB each) or 7 of 128 (28 KB
    // each), leaving room for a charge-spreading CTA beside them
    const int reserve = (shape & 1) ? ((shape & 2) ? 28 * 1024 : 60 * 1024) : 0;
    static std::atomic<unsigned long long> attr{0ull};
    once_per_device(attr, [] {
        cudaFuncSetAttribute(k_nonbonded<ES, 0, false, false, SP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             90 * 1024);
        cudaFuncSetAttribute(k_nonbonded<ES, 0, true, false, SP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             90 * 1024);
    });
    if (shape & 4) k_nonbonded<ES, 0, true, false, SP><<<grid, tb, reserve, s>>>(st, p);
    else k_nonbonded<ES, 0, false, false, SP><<<grid, tb, reserve, s>>>(st, p);
}

template <int ES>
static void launch_nb_plain(const DevState& st, const NbParams& p, bool energy, int shape, cudaStream_t s) {
    if (st.nb_split) launch_nb_shape<ES, true>(st, p, energy, shape, s);
    else launch_nb_shape<ES, false>(st, p, energy, shape, s);
}

int launch_nonbonded(const DevState& st, const NbParams& p, bool energy, cudaStream_t s, int shape) {
    // the staged kernel takes whole clusters: with rows split over warps, its
    // shapes run the plain kernel's matching shape (the same bits either way)
    if ((shape & 8) && st.nb_split) shape &= 7;
    if (shape & 8) {
        if (p.es_mode == 0) launch_nb_staged<0>(st, p, energy, shape, s);
        else if (p.es_mode == 1) launch_nb_staged<1>(st, p, energy, shape, s);
        else launch_nb_staged<2>(st, p, energy, shape, s);
        return 1;
    }
    if (p.es_mode == 0) launch_nb_plain<0>(st, p, energy, shape, s);
    else if (p.es_mode == 1) launch_nb_plain<1>(st, p, energy, shape, s);
    else launch_nb_plain<2>(st, p, energy, shape, s);
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
        for (int k = 0; k < 3; ++k) d[k] -= sd.box[k] * rint(d[k] * sd.inv_box[k]);
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
            if (st.atom_energy) {
                add_atom_energy(st.epot, si, 0.5 * e);
                add_atom_energy(st.epot, sj, 0.5 * e);
            }
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

// The reference's immediate-neighbour pairs (reference convention with
// compounds): every pair inside one compound or across two bonded compounds,
// minus the excluded pairs, evaluated with NO cutoff
// (compoundImmediateneighborAndSelfShortrangeInteractionsKernel,
// EngineKernels.cuh:150-317, through the LUT overload of
// computeCompoundCompoundLJForces, LennardJonesInteractions.cuh:121-161).  The
// same LJ and real-space Coulomb arithmetic as the pair kernel (sigma/2 and
// sqrt(eps) per atom, erfc(kappa r) in Ewald mode); the EM variant clamps the LJ
// force as the reference's energy minimiser does.  One thread per pair; the
// difference vector comes from the FP64 positions with the minimum image.
template <bool ENERGY>
__global__ void k_immediate_pairs(DevState st, BondedTerms bt, NbParams p) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double elj = 0.0, ecl = 0.0, vir = 0.0;
    int sysi = -1;
    if (t < bt.nm) {
        const int2 pr = bt.midx[t];
        const int si = st.slot_of[pr.x], sj = st.slot_of[pr.y];
        sysi = st.atom_sys[pr.x];
        const SysDesc& sd = st.sys[sysi];
        double d[3] = {st.px[sj] - st.px[si], st.py[sj] - st.py[si], st.pz[sj] - st.pz[si]};   // r_j - r_i
        if (st.periodic)
            for (int k = 0; k < 3; ++k) d[k] -= sd.box[k] * rint(d[k] * sd.inv_box[k]);
        const float dx = (float)d[0], dy = (float)d[1], dz = (float)d[2];
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float rinv = rsqrtf(r2);
        const float rinv2 = rinv * rinv;
        const float2 li = st.ljp[si], lj = st.ljp[sj];
        const float sig = li.x + lj.x, eps = li.y * lj.y;
        float s6 = sig * sig * rinv2;
        s6 = s6 * s6 * s6;
        // attraction along r_j - r_i when positive
        float fs = 24.f * eps * s6 * rinv2 * (1.f - 2.f * s6);
        if (p.em) fs = em_lj_clamp(fs, r2 * rinv);
        const float qq = p.ke * st.xyzq[si].w * st.xyzq[sj].w;
        float ec = 0.f;
        if (p.es_mode != 0 && qq != 0.f) {
            float fc = qq * rinv * rinv2;   // repulsion along r_i - r_j
            ec = qq * rinv;
            if (p.es_mode == 2) {
                const float r = r2 * rinv, kr = p.kappa * r;
                const float erfc_kr = erfcf(kr);
                fc *= erfc_kr + p.two_kappa_sqrtpi * r * __expf(-kr * kr);
                ec *= erfc_kr;
            }
            fs -= fc;
        }
        if (p.em) fs = fmaxf(fminf(fs, 1e20f), -1e20f);
        const float fx = fs * dx, fy = fs * dy, fz = fs * dz;   // force on i
        atomic_add_fixed(st.fx + si, to_fixed(fx, FORCE_SCALE));
        atomic_add_fixed(st.fy + si, to_fixed(fy, FORCE_SCALE));
        atomic_add_fixed(st.fz + si, to_fixed(fz, FORCE_SCALE));
        atomic_add_fixed(st.fx + sj, to_fixed(-fx, FORCE_SCALE));
        atomic_add_fixed(st.fy + sj, to_fixed(-fy, FORCE_SCALE));
        atomic_add_fixed(st.fz + sj, to_fixed(-fz, FORCE_SCALE));
        if (ENERGY) {
            elj = 4.0 * (double)eps * (double)s6 * ((double)s6 - 1.0);
            ecl = (double)ec;
            vir = 0.5 * (double)fs * (double)r2;   // -1/2 r_ij . f_ij
            if (st.atom_energy) {
                add_atom_energy(st.epot, si, 0.5 * (elj + ecl));
                add_atom_energy(st.epot, sj, 0.5 * (elj + ecl));
            }
        }
    }
    if (ENERGY) {
        add_energy_fixed(st.energy, sysi, elj, E_LJ);
        add_energy_fixed(st.energy, sysi, ecl, E_COUL);
        add_energy_fixed(st.energy, sysi, vir, E_VIRIAL);
    }
}

int launch_immediate_pairs(const DevState& st, const BondedTerms& bt, const NbParams& p, bool energy,
                           cudaStream_t s) {
    if (bt.nm == 0) return 0;
    const int TB = 256;
    if (energy)
        k_immediate_pairs<true><<<(bt.nm + TB - 1) / TB, TB, 0, s>>>(st, bt, p);
    else
        k_immediate_pairs<false><<<(bt.nm + TB - 1) / TB, TB, 0, s>>>(st, bt, p);
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
    const int n = min(st.walk_count[ci], st.pl_cap);
    const int sysi = st.cluster_sys[ci];
    const float Lx = st.sys[sysi].boxf[0], Ly = st.sys[sysi].boxf[1], Lz = st.sys[sysi].boxf[2];
    const size_t base = (size_t)ci * st.pl_cap;
    for (int k = lane; k < n; k += 32) {
        const int2 row = st.walk_row[base + k];
        const int sj = row.x;
        const unsigned img = (unsigned)row.y >> ROW_SHIFT_BIT;
        const int3 sh = make_int3((int)(img & 3u) - 1, (int)((img >> 2) & 3u) - 1, (int)(img >> 4) - 1);
        const float4 xj = st.xyzq[sj];
        for (int ii = 0; ii < CLUSTER; ++ii) {
            const float4 xi = st.xyzq[ci * CLUSTER + ii];
            const float dx = xj.x + sh.x * Lx - xi.x;
            const float dy = xj.y + sh.y * Ly - xi.y;
            const float dz = xj.z + sh.z * Lz - xi.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (((row.y >> ii) & 1) && r2 <= p.rc2) {
                const int ai = st.orig[ci * CLUSTER + ii];
                const int aj = st.orig[sj];
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
