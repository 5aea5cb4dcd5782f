// bonded.cu — bonds, angles (+Urey-Bradley), proper dihedrals, impropers and
// LJ pair bonds, one thread per term.
//
// Replaces BondgroupsKernel (code/LIMA_ENGINE/src/EngineKernels.cuh:716-823) and
// the term functions of code/LIMA_ENGINE/src/ForceComputations.cuh:
//   calcSinglebondForces :17-51, calcAnglebondForces :53-115,
//   calcDihedralbondForces :119-210, calcImproperdihedralbondForces :214-264,
//   computePairbondForces :335-376.
// The reference serialises per-atom accumulation through a 64-thread loop with
// a __syncthreads per term (ForceComputations.cuh:317-325) to be deterministic;
// here each term adds its forces as int64 fixed point, which is order-free.
// Vectors inside a term are FP64 differences of the master positions (minimum
// image), rounded to FP32 for the term arithmetic.
#include "engine.h"

namespace lima {

namespace {
struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float len(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 unit(f3 a) {
    const float l = len(a);
    return l > 0.f ? a * (1.f / l) : f3{0.f, 0.f, 0.f};
}

// position of atom a relative to atom a0 (FP64 difference; minimum image in a periodic box)
__device__ __forceinline__ f3 rel(const DevState& st, const SysDesc& sd, int s0, int a) {
    const int s = st.slot_of[a];
    double d[3] = {st.px[s] - st.px[s0], st.py[s] - st.py[s0], st.pz[s] - st.pz[s0]};
    if (st.periodic) {
#pragma unroll
        for (int k = 0; k < 3; ++k) d[k] -= sd.box[k] * rint(d[k] * sd.inv_box[k]);
    }
    return {(float)d[0], (float)d[1], (float)d[2]};
}

__device__ __forceinline__ void add_force(const DevState& st, int a, f3 f) {
    const int s = st.slot_of[a];
    atomic_add_fixed(st.fx + s, to_fixed(f.x, FORCE_SCALE));
    atomic_add_fixed(st.fy + s, to_fixed(f.y, FORCE_SCALE));
    atomic_add_fixed(st.fz + s, to_fixed(f.z, FORCE_SCALE));
}

// harmonic bond: E = kb/2 (|d|-b0)^2, force on a along -d
__device__ __forceinline__ float bond_term(f3 d /* a - b */, float b0, float kb, f3* f) {
    const float r = len(d);
    const float err = r - b0;
    const f3 u = unit(d);
    f[0] = u * (-kb * err);
    f[1] = u * (kb * err);
    return 0.5f * kb * err * err;
}

// harmonic angle on in-plane normals + Urey-Bradley spring (positions relative to the middle atom)
__device__ __forceinline__ float angle_term(f3 a1 /* l - m */, f3 a2 /* r - m */, float4 par, f3* f) {
    const f3 v1 = unit(a1), v2 = unit(a2);
    const f3 nrm = unit(cross(v1, v2));
    const f3 dl = unit(cross(nrm, v1));
    const f3 dr = unit(cross(v2, nrm));
    const float c = fminf(1.f, fmaxf(-1.f, dot(v1, v2)));
    const float err = acosf(c) - par.x;
    const float torque = par.y * err;
    f[0] = dl * (torque / len(a1));
    f[2] = dr * (torque / len(a2));
    f[1] = (f[0] + f[2]) * -1.f;
    float e = 0.5f * par.y * err * err;
    const f3 d13 = a1 - a2;
    const float e13 = len(d13) - par.z;
    const f3 u13 = unit(d13);
    f[0] = f[0] + u13 * (-par.w * e13);
    f[2] = f[2] + u13 * (par.w * e13);
    e += 0.5f * par.w * e13 * e13;
    return e;
}

// periodic dihedral k(1+cos(n tau - phi0)), tau = -atan2(sin phi, cos phi)
__device__ __forceinline__ float dihedral_term(f3 b1, f3 b2, f3 b3, float4 par, f3* f) {
    const float phi0 = par.x, k = par.y, mult = par.z;
    const f3 A = cross(b1, b2), B = cross(b2, b3), C = cross(b2, A);
    const float iA = 1.f / len(A), iB = 1.f / len(B), iC = 1.f / len(C);
    const float cphi = dot(A, B) * iA * iB;
    const float sphi = dot(C, B) * iC * iB;
    const float tau = -atan2f(sphi, cphi);
    const float e = k * (1.f + cosf(mult * tau - phi0));
    const float torque = k * mult * sinf(mult * tau - phi0);
    const f3 Bn = B * iB;
    f3 g1, g2, g3;
    if (fabsf(sphi) > 0.1f) {
        const f3 An = A * iA;
        const f3 dA = (An * cphi - Bn) * iA;
        const f3 dB = (Bn * cphi - An) * iB;
        const float s = torque / sphi;
        g1 = cross(b2, dA) * s;
        g3 = cross(b2, dB) * (-s);
        g2 = (cross(b3, dB) - cross(b1, dA)) * s;
    } else {
        const f3 Cn = C * iC;
        const f3 dC = (Cn * sphi - Bn) * iC;
        const f3 dB = (Bn * sphi - Cn) * iB;
        const float s = -torque / cphi;
        g1 = cross(b2, cross(dC, b2)) * s;
        g3 = cross(dB, b2) * s;
        const f3 t = b2 * (2.f * dot(b1, dC)) - b1 * dot(b2, dC) - dC * dot(b2, b1);
        g2 = (t + cross(b3, dB)) * s;
    }
    f[0] = g1;
    f[1] = g2 - g1;
    f[2] = g3 - g2;
    f[3] = g3 * -1.f;
    return e;
}

__device__ __forceinline__ float dist_to_line(f3 p, f3 a, f3 b) {
    return len(cross(b - a, a - p)) / len(b - a);
}

// improper: signed angle between the (i,j,k) and (l,j,k) planes
__device__ __forceinline__ float improper_term(f3 pi, f3 pj, f3 pk, f3 pl, float2 par, f3* f) {
    const f3 ij = unit(pj - pi), ik = unit(pk - pi), il = unit(pl - pi);
    const f3 lj = unit(pj - pl), lk = unit(pk - pl);
    const f3 n1 = unit(cross(ij, ik));
    const f3 n2 = unit(cross(lj, lk));
    float ang = acosf(fminf(1.f, fmaxf(-1.f, dot(n1, n2))));
    if (dot(n1, il) > 0.f) ang = -ang;
    const float err = ang - par.x;
    const float torque = par.y * err;
    f[3] = n2 * (torque / dist_to_line(pl, pj, pk));
    f[0] = n1 * (-torque / dist_to_line(pi, pj, pk));
    const f3 rest = (f[0] + f[3]) * -1.f;
    const float lij = len(pj - pi), lik = len(pk - pi);
    const float ratio = lij / (lij + lik);
    f[1] = rest * (1.f - ratio);
    f[2] = rest * ratio;
    return 0.5f * par.y * err * err;
}

// LJ pair bond, no cutoff; d = b - a
__device__ __forceinline__ float pairbond_term(f3 d, float sig, float eps, f3* f) {
    const float r2 = dot(d, d);
    float s = sig * sig / r2;
    s = s * s * s;
    const float fs = 24.f * eps * s / r2 * (1.f - 2.f * s);
    f[0] = d * fs;
    f[1] = d * (-fs);
    return 4.f * eps * s * (s - 1.f);
}
}  // namespace

template <bool ENERGY>
__global__ void k_bonded(DevState st, BondedTerms bt) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = bt.nb + bt.na + bt.nd + bt.ni + bt.np;
    float en = 0.f, vir = 0.f;   // this thread's term energy (of kind `kind`) and virial
    int sysi = -1, kind = -1;
    if (t < total) {
        f3 f[4];
        f3 r[4];
        int atoms[4];
        int na = 0;
        kind = 0;
        if (t < bt.nb) {
            const int2 ix = bt.bidx[t];
            atoms[0] = ix.x;
            atoms[1] = ix.y;
            na = 2;
            kind = 0;
        } else if ((t -= bt.nb) < bt.na) {
            const int4 ix = bt.aidx[t];
            atoms[0] = ix.x;
            atoms[1] = ix.y;
            atoms[2] = ix.z;
            na = 3;
            kind = 1;
        } else if ((t -= bt.na) < bt.nd) {
            const int4 ix = bt.didx[t];
            atoms[0] = ix.x;
            atoms[1] = ix.y;
            atoms[2] = ix.z;
            atoms[3] = ix.w;
            na = 4;
            kind = 2;
        } else if ((t -= bt.nd) < bt.ni) {
            const int4 ix = bt.iidx[t];
            atoms[0] = ix.x;
            atoms[1] = ix.y;
            atoms[2] = ix.z;
            atoms[3] = ix.w;
            na = 4;
            kind = 3;
        } else {
            t -= bt.ni;
            const int2 ix = bt.pidx[t];
            atoms[0] = ix.x;
            atoms[1] = ix.y;
            na = 2;
            kind = 4;
        }
        sysi = st.atom_sys[atoms[0]];
        const SysDesc& sd = st.sys[sysi];
        const int s0 = st.slot_of[atoms[0]];
        // loops over the term's atoms run to 4 with a guard, so that every index is
        // a constant and atoms, r and f stay in registers
        r[0] = f3{0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 1; k < 4; ++k)
            if (k < na) r[k] = rel(st, sd, s0, atoms[k]);
        switch (kind) {
            case 0: {
                const float2 p = bt.bpar[t];
                en = bond_term(r[0] - r[1], p.x, p.y, f);
            } break;
            case 1:
                en = angle_term(r[0] - r[1], r[2] - r[1], bt.apar[t], f);
                break;
            case 2:
                en = dihedral_term(r[1] - r[0], r[2] - r[1], r[3] - r[2], bt.dpar[t], f);
                break;
            case 3:
                en = improper_term(r[0], r[1], r[2], r[3], bt.ipar[t], f);
                break;
            default: {
                const float2 p = bt.ppar[t];
                en = pairbond_term(r[1] - r[0], p.x, p.y, f);
            } break;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < na) {
                add_force(st, atoms[k], f[k]);
                if (ENERGY) {
                    vir += -0.5f * dot(r[k], f[k]);
                    if (st.atom_energy) add_atom_energy(st.epot, st.slot_of[atoms[k]], (double)en / na);  // equal shares
                }
            }
        }
    }
    if (ENERGY) {
        const int terms[5] = {E_BOND, E_ANGLE, E_DIHEDRAL, E_IMPROPER, E_PAIRBOND};
        // terms are stored kind by kind, so a warp almost always holds one kind:
        // then only that kind's total (and the virial) needs a warp sum
        const int k0 = __reduce_max_sync(0xffffffffu, kind);
        if (__all_sync(0xffffffffu, kind < 0 || kind == k0)) {
            if (k0 >= 0) add_energy_fixed(st.energy, sysi, kind >= 0 ? (double)en : 0.0, terms[k0]);
        } else {
#pragma unroll
            for (int k = 0; k < 5; ++k) add_energy_fixed(st.energy, sysi, kind == k ? (double)en : 0.0, terms[k]);
        }
        add_energy_fixed(st.energy, sysi, (double)vir, E_VIRIAL);
    }
}

int launch_bonded(const DevState& st, const BondedTerms& bt, bool energy, cudaStream_t s) {
    const int total = bt.nb + bt.na + bt.nd + bt.ni + bt.np;
    if (total == 0) return 0;
    const int TB = 128;
    if (energy)
        k_bonded<true><<<(total + TB - 1) / TB, TB, 0, s>>>(st, bt);
    else
        k_bonded<false><<<(total + TB - 1) / TB, TB, 0, s>>>(st, bt);
    return 1;
}

}  // namespace lima
