// common.cuh — device-side layout shared by every kernel of the force and
// integration path.
//
// Data layout in HBM (all systems of a batch concatenated):
//   * atoms live in "slots": the spatially sorted order produced by the
//     column/cluster binning.  Slot s belongs to cluster s/8; padding slots
//     have orig[s] == -1, zero charge/LJ and zero inverse mass.
//   * per-slot state: pos (FP64 x,y,z SoA), xyzq (float4 working copy),
//     ljp (float2: sigma/2, sqrt(eps)), vel (float4: v, 1/m), fprev (float4),
//     force accumulators f{x,y,z} (int64 fixed point, FORCE_SCALE per J/mol/nm)
//   * per-system energy accumulators: int64 fixed point, ENERGY_SCALE per J/mol
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lima {

constexpr int CLUSTER = 8;                       // atoms per cluster
constexpr double FORCE_SCALE = 4294967296.0;     // 2^32 per J/mol/nm
constexpr double ENERGY_SCALE = 16777216.0;      // 2^24 per J/mol
constexpr double GRID_SCALE = 1099511627776.0;   // 2^40 per kC/mol (int64 PME charge grid)
// the engine's int32 PME charge grid: 2^20 per kC/mol, so a node holds up to
// +-2048 kC/mol (about 21 e of B-spline-weighted charge) in steps of 1e-8 e
constexpr double GRID32_SCALE = 1048576.0;
constexpr int SHIFT_BITS = 5;                    // periodic-shift code in the pair search's candidates
constexpr int JCLUSTER_BITS = 32 - SHIFT_BITS;

enum EnergyTerm {
    E_LJ = 0, E_COUL, E_RECIP, E_SELF, E_EXCL, E_BOND, E_ANGLE, E_DIHEDRAL, E_IMPROPER,
    E_PAIRBOND, E_KINETIC, E_VIRIAL, E_COUNT
};

// status word bits (mirror LIMA_STATUS_* in include/lima_b200.h)
constexpr unsigned ST_PAIRLIST_OVERFLOW = 0x1u;
constexpr unsigned ST_COLUMN_OVERFLOW = 0x2u;
constexpr unsigned ST_NONFINITE = 0x4u;
constexpr unsigned ST_FORCE_SATURATED = 0x8u;
constexpr unsigned ST_MOVED_TOO_FAR = 0x10u;

// Per-system descriptor (one per system of a batch), resident in global memory.
struct SysDesc {
    double box[3];        // [nm]
    double inv_box[3];    // 1 / box
    float boxf[3];
    float inv_boxf[3];
    int atom_off, n_atoms;          // original-order atom range
    int col_off, ncol_x, ncol_y;    // column grid
    float col_w[2];                 // column widths [nm]
    int max_clusters;               // capacity of this system's cluster range
    int cluster_cap_off;            // first cluster of this system's capacity range
    int pme_off;                    // offset of the real PME grid (floats)
    int pme_coff;                   // offset of the half-complex grid (float2)
    int pme_n[3];                   // grid dims (0 = no PME)
    float pme_inv_h[3];             // K_d / L_d
    double self_energy;             // Ewald self term [J/mol]
    int n_charged;
    float self_coef;                // per-atom self energy: self_coef * q^2, or self_coef per
    int self_per_charge;            //   charged atom when self_per_charge (reference convention)
    float efield[3];                // uniform external field x 1000: force = q [kC/mol] x efield [J/mol/nm]
    int nb_parts;                   // pair-kernel warps per i-cluster (its rows split in 32-row multiples)
    int pad_;
};

// scale is a power of two, so v * (float)scale is exact and one float->int64
// conversion gives the same integer as rounding (double)v * scale
__device__ __forceinline__ long long to_fixed(float v, double scale) {
    return __float2ll_rn(v * (float)scale);
}
__device__ __forceinline__ long long to_fixed_d(double v, double scale) {
    return __double2ll_rn(v * scale);
}
__device__ __forceinline__ void atomic_add_fixed(long long* p, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

__device__ __forceinline__ float min_image(float d, float L, float invL) {
    return d - L * rintf(d * invL);
}

// warp reduction of a double (fixed lane order, so bit-reproducible)
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Adds one lane's energy contribution to system `sysi`'s accumulator.  Each
// lane's value is rounded to fixed point first and the warp sums integers, so
// the total does not depend on how lanes are grouped into warps (a system run
// alone and the same system inside a batch give identical bits).
__device__ __forceinline__ void add_energy_fixed(long long* energy, int sysi, double e, int term) {
    const long long v = sysi >= 0 ? __double2ll_rn(e * ENERGY_SCALE) : 0ll;
    const int s0 = __shfl_sync(0xffffffffu, sysi, 0);
    const bool uniform = __all_sync(0xffffffffu, sysi == s0 || sysi < 0);
    const int sref = __reduce_max_sync(0xffffffffu, sysi);
    if (uniform) {
        const long long t = warp_sum_ll(v);
        if ((threadIdx.x & 31) == 0 && sref >= 0)
            atomicAdd(reinterpret_cast<unsigned long long*>(energy + (size_t)sref * E_COUNT + term),
                      static_cast<unsigned long long>(t));
    } else if (sysi >= 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(energy + (size_t)sysi * E_COUNT + term),
                  static_cast<unsigned long long>(v));
    }
}

// adds an atom's share of a potential energy [J/mol] to its per-slot accumulator
// (fixed point, ENERGY_SCALE per J/mol; each share is rounded before the add,
// so the per-atom sums do not depend on the order of the adds)
__device__ __forceinline__ void add_atom_energy(long long* epot, int slot, double e) {
    atomicAdd(reinterpret_cast<unsigned long long*>(epot + slot),
              static_cast<unsigned long long>(__double2ll_rn(e * ENERGY_SCALE)));
}

// shift code (sx+1) + 3(sy+1) + 9(sz+1), s in {-1,0,1}
__device__ __forceinline__ int3 decode_shift(int code) {
    return make_int3(code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1);
}

}  // namespace lima
