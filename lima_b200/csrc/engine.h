// engine.h — internal host/device interface of the force and integration path.
// Not part of the public C-ABI (include/lima_b200.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>

#include "common.cuh"

namespace lima {

// Kernel attributes (the dynamic shared-memory limit) belong to one device's
// context.  Runs set_attributes once per device (bit d of `done` for device d):
// under a lock, and the bit is published only after set_attributes returns, so
// a second host thread driving another engine on the same device never
// launches before the attributes are in place.
template <class F>
inline void once_per_device(std::atomic<unsigned long long>& done, F&& set_attributes) {
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (done.load(std::memory_order_relaxed) & bit) return;
    set_attributes();
    done.fetch_or(bit, std::memory_order_release);
}

// Every device pointer the per-step kernels touch; passed to kernels by value.
struct DevState {
    int n_sys = 0;
    int n_atoms = 0;          // all systems
    int n_clusters = 0;       // capacity (sum of per-system max_clusters)
    int n_slots = 0;          // 8 * n_clusters
    int n_cols = 0;           // all columns
    int pl_cap = 0;           // pair-list rows per i-cluster
    int atom_energy = 0;      // energy evaluations also add per-atom shares to epot (log frames)
    int has_field = 0;        // some system has an external field: forces start from q E, not zero
    int periodic = 1;         // 0: no boundary condition (no images, no wrapping, plain differences)
    int col_cap = 0;          // atoms a column may hold
    // pair-kernel warps: system s owns warps [nb_warp_off[s], nb_warp_off[s + 1]),
    // max_clusters x nb_parts of them; nb_split: some system has nb_parts > 1
    int nb_warps = 0;
    int nb_split = 0;
    const int* nb_warp_off = nullptr;

    SysDesc* sys = nullptr;
    int* sys_nclusters = nullptr;   // actual clusters per system (device-written)
    int* cluster_sys = nullptr;     // static: system of each cluster slot range
    int* col_sys = nullptr;         // static: system of each column

    // per-slot state
    double *px = nullptr, *py = nullptr, *pz = nullptr;
    float4* xyzq = nullptr;
    float2* ljp = nullptr;          // sigma/2, sqrt(eps)
    float4* vel = nullptr;          // v, 1/m
    float4* fprev = nullptr;        // previous-step force (velocity Verlet)
    float4* adam_m = nullptr;       // energy minimisation first moments
    float4* adam_v = nullptr;       // second moments
    long long *fx = nullptr, *fy = nullptr, *fz = nullptr;
    int* orig = nullptr;
    int* slot_mol = nullptr;        // molecule id per slot (-1 for padding)
    float4* tvel = nullptr;         // permutation scratch
    float4* tfprev = nullptr;
    float4* tadam_m = nullptr;
    float4* tadam_v = nullptr;

    // per-atom (original order), static
    int* atom_sys = nullptr;
    int* slot_of = nullptr;
    float* q = nullptr;
    float* inv_mass = nullptr;
    float2* ljp_atom = nullptr;
    int* mol = nullptr;
    int* excl_off = nullptr;
    int* excl_idx = nullptr;
    double* in_pos = nullptr;       // 3n staging / wrapped positions
    float* in_vel = nullptr;        // 3n staging

    // binning scratch
    int* col_of_atom = nullptr;
    float* z_of_atom = nullptr;
    int* col_count = nullptr;
    int* col_fill = nullptr;
    int* col_atom_start = nullptr;
    int* col_cl_start = nullptr;
    int* col_ncl = nullptr;
    int* col_list = nullptr;
    int* new_orig = nullptr;

    // clusters and pair list
    float4* bb_lo = nullptr;
    float4* bb_hi = nullptr;
    unsigned long long* bb_molsig = nullptr;  // bit (molecule id mod 64) of every atom in the cluster
    int* pl_count = nullptr;
    // pair-list rows: one per (i-cluster, j-atom) with at least one i-atom in range;
    // x = j slot, y = 8-bit i-atom mask | periodic shift code << 8
    int2* pl_row = nullptr;
    // the inner list: the rows of pl_row still within r_in of one of their
    // i-atoms at the last prune (k_prune_rows), same format and capacity
    int* pl_count_in = nullptr;
    int2* pl_row_in = nullptr;
    // the list the pair kernels walk: pl_row/pl_count after a rebuild, the
    // inner list after a prune
    const int* walk_count = nullptr;
    const int2* walk_row = nullptr;
    int* nb_counter = nullptr;      // next i-cluster of the persistent (staged) pair kernel
    // split pair search (nb_split): warp w of the search writes its rows to
    // ps_stage[w * pl_cap ...] and their count to ps_stage_count[w]; a second
    // kernel concatenates each cluster's parts in order into pl_row
    int2* ps_stage = nullptr;
    int* ps_stage_count = nullptr;

    // PME
    int* pme_grid_fx = nullptr;          // fixed-point charge grid, GRID32_SCALE (all systems)
    float* pme_real = nullptr;           // real-space potential grid
    float2* pme_cplx = nullptr;          // half-complex grid
    float* pme_theta = nullptr;          // influence function on the half-complex grid
    float2* pme_tw = nullptr;            // twiddle tables e^{-2 pi i k/n} for every grid length
    int pme_total_real = 0;
    int pme_total_cplx = 0;

    unsigned* status = nullptr;
    long long* energy = nullptr;         // [n_sys][E_COUNT]
    long long* epot = nullptr;           // per-slot potential energy (energy steps), fixed point
    float4* xyz_ref = nullptr;           // per-slot position at the last pair-list build
    float* vscale = nullptr;             // per-system velocity scale of the integrator (thermostat)
};

struct BondedTerms {
    int nb = 0, na = 0, nd = 0, ni = 0, np = 0;
    int2* bidx = nullptr;
    float2* bpar = nullptr;
    int4* aidx = nullptr;
    float4* apar = nullptr;
    int4* didx = nullptr;
    float4* dpar = nullptr;
    int4* iidx = nullptr;
    float2* ipar = nullptr;
    int2* pidx = nullptr;
    float2* ppar = nullptr;
    int nx = 0;                 // excluded charged pairs for the Ewald correction
    int2* xidx = nullptr;
    int nm = 0;                 // immediate-neighbour pairs (ref_compat compounds): no cutoff
    int2* midx = nullptr;
};

// p of the Abramowitz & Stegun 7.1.26 erfc form the pair kernel uses
constexpr float AS_P = 0.3275911f;
struct NbParams {
    float rc2;
    float rlist;          // cutoff + skin
    int es_mode;          // 0 none, 1 cutoff, 2 Ewald erfc
    float kappa;
    float ke;             // Coulomb constant
    float two_kappa_sqrtpi;
    float mk2_log2e;      // -kappa^2 log2(e): exp(-kappa^2 r^2) = 2^(mk2_log2e r^2)
    float p_kappa;        // AS_P kappa: the pair kernel's erfc takes t = 1/(1 + p kappa r)
    int em;               // energy minimisation: force-only launches take the pair kernel's EM variant
};
// periodic image of a pair-list row: (sx + 1) | (sy + 1) << 2 | (sz + 1) << 4 in bits
// 8-13 of the row's second word, above the 8-bit i-mask
constexpr int ROW_SHIFT_BIT = 8;

// nbsearch.cu
int launch_rebuild(const DevState& st, float rlist, bool from_input, cudaStream_t s);
int launch_rebuild_slots(const DevState& st, bool from_input, cudaStream_t s);   // stages 1-7
int launch_pairsearch(const DevState& st, float rlist, cudaStream_t s);          // stage 8
// the inner list at radius rin from the current positions (rows of the outer list)
int launch_prune(const DevState& st, float rin, cudaStream_t s);
// nonbonded.cu
// shape: launch shape of the force-only kernel (bit 0 residency cap, bit 1 128-thread blocks)
int launch_nonbonded(const DevState& st, const NbParams& p, bool energy, cudaStream_t s, int shape = 0);
int launch_exclusion_correction(const DevState& st, const BondedTerms& bt, const NbParams& p,
                                 bool energy, cudaStream_t s);
int launch_pairlist_dump(const DevState& st, const NbParams& p, long long cap, int* out_pairs,
                          unsigned long long* out_count, cudaStream_t s);
int launch_immediate_pairs(const DevState& st, const BondedTerms& bt, const NbParams& p, bool energy,
                           cudaStream_t s);
// bonded.cu
int launch_bonded(const DevState& st, const BondedTerms& bt, bool energy, cudaStream_t s);
// pme.cu
constexpr int PME_FFT_TX = 16;       // half-complex columns per CTA of the y and z passes
constexpr int PME_FFT_XLINES = 8;    // lines per CTA of the x passes
struct PmePlan {
    int n_items_x = 0, n_items_y = 0, n_items_z = 0;   // work items per FFT pass
    int4* items_x = nullptr;     // (system, line0, nlines, 0)
    int4* items_y = nullptr;     // (system, x0, z, 0)
    int4* items_z = nullptr;     // (system, x0, y, 0)
    const void* sys_plans = nullptr;  // per-system radix plans (device)
    int ref_gather = 0;          // central-difference gather
    int max_n = 0;
    // plane-fused x+y passes (one CTA per z-plane), used when every plane fits
    // in shared memory; otherwise the separate x and y passes run
    int n_items_xy = 0;
    int4* items_xy = nullptr;    // (system, z, 0, 0)
    int xy_buf = 0;              // float2 elements per ping-pong buffer
    // charge spreading by column blocks (one CTA per item, a shared-memory box
    // of grid nodes per CTA); none when a box would not fit
    int n_items_spread = 0;
    int4* items_spread = nullptr;   // (system, first column x, first column y, first z node)
    int4* spread_geo = nullptr;     // per system: box nodes in x, y, z (0 = no grid)
    int spread_box = 0;             // int32 elements of the largest box
    int n_sys = 0;                  // systems of the plan; with one, its descriptor
    SysDesc sys0{};                 //   travels as a kernel argument
};
constexpr int PME_SPREAD_COLS = 1;      // columns per block side
// int32 nodes of a box (40 KB of shared memory): small enough for a 256-thread
// spreading CTA to fit beside the pair kernel's CTAs on an SM, which the
// higher-priority PME stream relies on to overlap the two
constexpr int PME_SPREAD_MAX_BOX = 10240;
// nodes of a block's box along x or y: the block's width in grid units plus the
// order-4 stencil (atoms that drifted out of their column use the direct route)
int pme_spread_box_side(double col_w, double inv_h);
// shared-memory elements of one buffer of the plane-fused x+y passes for a
// K0 x K1 plane (0 = does not fit)
int pme_xy_buffer(int k0, int k1);
size_t pme_sys_dev_size();
bool fill_pme_sys_dev(void* dst, int kx, int ky, int kz);
void set_pme_sys_twiddles(void* dst, int offx, int offy, int offz);
void pme_set_smem_limits(int maxn, int xy_buf);
int launch_pme(const DevState& st, const PmePlan& plan, bool energy, cudaStream_t s);
// integrate.cu
struct IntegrateParams {
    double dt;
    int integrator;         // 0 leapfrog, 1 velocity Verlet (velocity scale: DevState::vscale)
    float half_skin2;       // (Verlet buffer / 2)^2: a larger move since the list build is flagged
};
int launch_integrate(const DevState& st, const IntegrateParams& p, bool energy, cudaStream_t s);
int launch_em_step(const DevState& st, int step, float* max_force_out_dev, cudaStream_t s);
int launch_gather_state(const DevState& st, double* pos_out, float* vel_out, cudaStream_t s);
int launch_gather_forces(const DevState& st, double* f_out, cudaStream_t s);
int launch_zero_forces(const DevState& st, cudaStream_t s);
int launch_max_force(const DevState& st, float* out, cudaStream_t s);
// per-system kinetic energy (E_KINETIC of ke[n_sys][E_COUNT], fixed point)
int launch_kinetic(const DevState& st, long long* ke, cudaStream_t s);
// new positions and velocities (original order, in_pos / in_vel) for atoms
// [a0, a0 + n) written into their current slots; the largest squared move from
// the last pair-list build goes to *max_disp2 (float bits, atomic max)
int launch_check_state(const DevState& st, int a0, int n, unsigned* word2, cudaStream_t s);
int launch_load_state(const DevState& st, int a0, int n, cudaStream_t s);
// one log frame in original atom order: (x, y, z, potential energy), (F, |v|)
int launch_log_frame(const DevState& st, float4* pos_epot, float4* force_speed, cudaStream_t s);

}  // namespace lima
