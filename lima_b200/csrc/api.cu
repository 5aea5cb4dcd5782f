// api.cu — the C-ABI (include/lima_b200.h) over the B200 force/integration path.
//
// Host-side equivalent of LIMA_ENGINE's Engine (code/LIMA_ENGINE/src/Engine.cu):
// construction uploads the system and builds the first pair list (Engine.cu:19-81),
// lima_step runs the per-step pipeline (_deviceMaster, Engine.cu:297-381, and the
// list rebuild of hostMaster, :161-190), readback replaces takeBackSim and the
// logging buffers.  Every entry point returns a LIMA_ERR_* code instead of
// throwing (code/LIMA_BASE/include/Utilities.h:22-51).
//
// Per step, on three streams joined by events:
//   main   : zero forces -> pair kernel ---------------------> integrate
//   bonded :        bonded terms + Ewald exclusion correction --^
//   pme    :        spread -> 5 FFT passes -> gather -----------^
#include <algorithm>
#include <climits>
#include <map>
#include <set>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "engine.h"
#include "lima_b200.h"
#include "mlp.h"

namespace {

using namespace lima;

constexpr double kCoulomb = 8.9875517873681764e9 / 1e-9 / 6.02214076e23 * 1000.0 * 1000.0;
constexpr double kPi = 3.14159265358979323846;
constexpr double kPiRef = 3.14159;  // code/LIMA_BASE/include/Constants.h:51

struct SystemHost {
    double box[3] = {0.0, 0.0, 0.0};
    int n = 0;
    std::vector<float> q, m, sig, eps;
    std::vector<int32_t> bonds, angles, dihedrals, impropers, pairbonds, excl;
    std::vector<float> bpar, apar, dpar, ipar, ppar;
    int pme[3] = {0, 0, 0};
    bool pme_set = false;
    std::vector<double> pos;
    std::vector<float> vel;
    double efield[3] = {0.0, 0.0, 0.0};   // external field [V/nm]
    std::vector<int32_t> compound;        // compound of each atom (-1: none); empty = not set
    std::vector<int32_t> bonded_compounds;  // pairs of bonded compound ids
};

struct CudaError {
    cudaError_t e;
    const char* what;
};

#define CK(x)                                            \
    do {                                                 \
        cudaError_t err__ = (x);                         \
        if (err__ != cudaSuccess) throw CudaError{err__, #x}; \
    } while (0)

struct ApiError {
    int code;
    std::string msg;
};

}  // namespace

struct lima_engine {
    lima_params p{};
    std::vector<SystemHost> sys;
    int cur = 0;
    std::string err;
    bool built = false;
    bool device_ok = false;   // set-up selected p.device successfully: calls select it again
    bool state_pending = false;
    int list_age = 1 << 30;
    int prune_every = 0;              // steps between prunes (0: no pruning)
    double rin = 0.0;                 // inner radius of the pruned list
    bool prune_pending = false;       // positions were handed in: prune before the next pair kernel
    int64_t step = 0;

    // derived
    double kappa = 0.0;
    double rlist = 0.0;
    bool pme_on = false;
    std::vector<double> self_energy;  // per system
    std::vector<int> n_atoms_off;

    DevState st{};
    BondedTerms bt{};
    PmePlan pp{};
    NbParams nb{};
    IntegrateParams ip{};
    std::vector<void*> allocs;
    cudaStream_t s_main = nullptr, s_bonded = nullptr, s_pme = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_bonded = nullptr, ev_pme = nullptr;
    cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;
    // phase timing: [rebuild, nonbonded, bonded, pme, integrate] x (start, stop)
    bool phase_timing = false;
    cudaEvent_t ev_ph[5][2] = {};
    double phase_ms[5] = {0, 0, 0, 0, 0};
    int phase_used[5] = {0, 0, 0, 0, 0};
    int64_t launches = 0;
    int64_t rebuilds = 0;
    // CUDA graph of one pair-list period: rebuild + nstlist (forces, integrate) steps
    cudaGraphExec_t graph_exec = nullptr;
    int64_t graph_launches_per_replay = 0;
    int64_t graph_replays = 0;

    // host mirrors
    std::vector<long long> energy_host;
    // pinned host words for the small read-backs that end a call (a copy to
    // pageable memory is staged and takes longer): [0, 2) status word and the
    // overflow count, [2, 4) the state hand-in's check words, then the energies
    unsigned* h_pin = nullptr;
    size_t h_pin_bytes = 0;
    unsigned last_status = 0;         // status word read at the end of the last run_steps
    long long* pin_energy() { return reinterpret_cast<long long*>(h_pin + 4); }
    bool energy_valid = false;
    double time_ms = 0.0;
    int64_t timed_steps = 0;

    // launch shape of the force-only pair kernel, picked by autotune()
    int nb_shape = 0;
    bool nb_tuned = false;
    double tune_ms[12] = {};   // per launch shape of the pair kernel

    // device scratch for readback
    unsigned* d_disp = nullptr;       // [0] largest squared move since the last list build (float bits),
                                      // [1] non-finite input flag
    int64_t state_fast_loads = 0;     // lima_set_state calls served without a rebuild
    double* d_out_d = nullptr;
    float* d_out_f = nullptr;
    float* d_maxf = nullptr;

    // thermostat (per system) and per-particle log
    long long* d_therm_ke = nullptr;   // [n_sys][E_COUNT]
    std::vector<double> therm_T, therm_scale;
    int64_t therm_step = -1;
    float4* log_pe = nullptr;          // device ring [log_ring][n_atoms]
    float4* log_fs = nullptr;
    int log_fill = 0;
    std::vector<int64_t> log_ring_steps;
    std::vector<float4> log_host_pe, log_host_fs;   // offloaded frames [frame][n_atoms]
    std::vector<int64_t> log_host_steps;

    // learned coarse-grid PME correction (mlp.cu, learned.cu)
    std::vector<SysDesc> sd_host;     // per-system descriptors of the engine's own grid
    bool lp_ready = false;            // buffers and model allocated
    bool lp_on = false;               // replaces the full-grid reciprocal part in stepping
    bool lp_fallback = false;         // a full-grid check failed: plain PME from then on
    bool lp_norm = false;             // input normalisation and output scale fixed
    bool lp_check_pending = false;
    int lp_check = 50;                // steps between full-grid checks
    double lp_tol = 1e-3;             // bound on the relative reciprocal-force RMSE
    double lp_last_rel = -1.0;
    int64_t lp_steps = 0;
    DevState st_c{};                  // view with the coarse grid, forces into lp_fc
    DevState st_f{};                  // view with the full grid, forces into lp_ff
    PmePlan pp_c{};
    long long* lp_fc = nullptr;       // coarse reciprocal force [3][n_slots]
    long long* lp_ff = nullptr;       // full-grid reciprocal force [3][n_slots]
    long long* lp_energy = nullptr;
    float* lp_feat = nullptr;         // [n_slots][68]
    __nv_bfloat16* lp_X = nullptr;    // [n_slots][80]
    float* lp_Y = nullptr;            // [n_slots][8]
    float* lp_mean = nullptr;
    float* lp_invstd = nullptr;
    MlpModel mlp{};
    MlpActs acts{};
    int batch_cap = 65536;
    __nv_bfloat16* batch_X = nullptr;
    float* batch_T = nullptr;
    float* batch_raw = nullptr;       // [batch_cap][68] staging of caller rows
    float* ds_feat = nullptr;         // collected frames, original atom order
    float* ds_target = nullptr;
    int ds_frames = 0;                // frames collected so far (ring of ds_cap)
    int ds_cap = 0;
    double* d_sums = nullptr;
    double* d_loss = nullptr;
    int* d_idx = nullptr;
    size_t d_idx_cap = 0;

    ~lima_engine() { release(); }

    template <typename T>
    T* dalloc(size_t n) {
        void* p_ = nullptr;
        if (n == 0) n = 1;
        CK(cudaMalloc(&p_, n * sizeof(T)));
        CK(cudaMemset(p_, 0, n * sizeof(T)));
        allocs.push_back(p_);
        return reinterpret_cast<T*>(p_);
    }
    template <typename T>
    T* upload(const std::vector<T>& v) {
        T* d = dalloc<T>(v.size());
        if (!v.empty()) CK(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        return d;
    }
    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
    void release() {
        if (s_main) cudaStreamSynchronize(s_main);
        drop_graph();
        for (void* a : allocs) cudaFree(a);
        allocs.clear();
        if (h_pin) cudaFreeHost(h_pin);
        h_pin = nullptr;
        h_pin_bytes = 0;
        for (cudaStream_t* s : {&s_main, &s_bonded, &s_pme})
            if (*s) cudaStreamDestroy(*s), *s = nullptr;
        for (cudaEvent_t* e : {&ev_fork, &ev_bonded, &ev_pme, &ev_t0, &ev_t1})
            if (*e) cudaEventDestroy(*e), *e = nullptr;
        for (auto& pr : ev_ph)
            for (cudaEvent_t& e : pr)
                if (e) cudaEventDestroy(e), e = nullptr;
        built = false;
        // the learned correction's buffers were among the allocations
        lp_ready = lp_on = lp_fallback = lp_norm = lp_check_pending = false;
        ds_frames = ds_cap = 0;
        d_idx = nullptr;
        d_idx_cap = 0;
        mlp = MlpModel{};
        acts = MlpActs{};
        log_fill = 0;
        log_ring_steps.clear();
    }

    void setup();
    void mark(int phase, int which, cudaStream_t s) {
        if (!phase_timing) return;
        CK(cudaEventRecord(ev_ph[phase][which], s));
        if (which == 1) phase_used[phase] = 1;
    }
    void collect_phases() {
        if (!phase_timing) return;
        CK(cudaDeviceSynchronize());
        for (int k = 0; k < 5; ++k) {
            if (!phase_used[k]) continue;
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ev_ph[k][0], ev_ph[k][1]));
            phase_ms[k] += ms;
            phase_used[k] = 0;
        }
    }
    PmePlan make_pme(std::vector<SysDesc>& sd, DevState& D);
    void rebuild(bool from_input);
    void start_rebuild(bool from_input);
    void finish_rebuild();
    bool begin_list();
    void rebuild_async();
    void forces(bool energy, bool atom_energy = false);
    void run_steps(int n);
    void capture_period();
    void read_energies(lima_energies* e);
    bool learned_active() const { return lp_ready && lp_on && !lp_fallback; }
    void learned_setup(int cx, int cy, int cz, int max_frames);
    void learned_features(bool forward, cudaStream_t s);
    void learned_full(cudaStream_t s, bool energy);
    void learned_pme_stage(bool energy, cudaStream_t s);
    void ensure_list();
    void measure_temperature();
    int autotune(int periods);
    void log_frame();
    void flush_log();
};

namespace {

int fail(lima_engine* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

template <typename F>
int guarded(lima_engine* h, F&& fn) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    // the current device is per host thread: a process may drive engines on
    // several devices, so every call works on its own engine's device
    if (h->device_ok) cudaSetDevice(h->p.device);
    try {
        return fn();
    } catch (const CudaError& e) {
        h->err = std::string("CUDA error in ") + e.what + ": " + cudaGetErrorString(e.e);
        return LIMA_ERR_CUDA;
    } catch (const ApiError& e) {
        h->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return LIMA_ERR_INVALID_ARG;
    }
}

double kappa_from_tol(double rc, double tol) {
    double lo = 0.0, hi = 20.0 / rc;
    for (int i = 0; i < 200; ++i) {
        const double mid = 0.5 * (lo + hi);
        if (std::erfc(mid * rc) > tol) lo = mid;
        else hi = mid;
    }
    return 0.5 * (lo + hi);
}

int fft_friendly(int n) {
    int m = std::max(n, 4);
    for (;; ++m) {
        int k = m;
        for (int p : {2, 3, 5})
            while (k % p == 0) k /= p;
        if (k == 1) return m;
    }
}

struct UnionFind {
    std::vector<int> p;
    explicit UnionFind(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
    int find(int x) {
        while (p[x] != x) x = p[x] = p[p[x]];
        return x;
    }
    void unite(int a, int b) {
        a = find(a);
        b = find(b);
        if (a != b) p[std::max(a, b)] = std::min(a, b);
    }
};

}  // namespace

void lima_engine::setup() {
    if (sys.empty()) throw ApiError{LIMA_ERR_STATE, "no systems"};
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        throw ApiError{LIMA_ERR_NO_DEVICE, "no CUDA device available"};
    CK(cudaSetDevice(p.device));
    device_ok = true;
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, p.device));
    if (prop.major < 10) throw ApiError{LIMA_ERR_NO_DEVICE, "this build targets sm_100a (B200)"};
    release();
    // frames logged under an earlier topology no longer match the atoms
    log_host_pe.clear();
    log_host_fs.clear();
    log_host_steps.clear();

    // ---- derived parameters
    const double rc = p.cutoff;
    if (!(rc > 0.0)) throw ApiError{LIMA_ERR_INVALID_ARG, "cutoff must be > 0"};
    const double skin = p.skin < 0.0 ? 0.1 : p.skin;
    rlist = rc + skin;
    if (p.nstlist < 1) throw ApiError{LIMA_ERR_INVALID_ARG, "nstlist must be >= 1"};
    if (p.electrostatics == LIMA_ES_EWALD) {
        if (p.ewald_kappa > 0.0) kappa = p.ewald_kappa;
        else if (p.ref_compat) kappa = 3.0 / rc;  // PhysicsUtils.cuh:60-62
        else kappa = kappa_from_tol(rc, p.ewald_tol > 0.0 ? p.ewald_tol : 1e-5);
    } else {
        kappa = 0.0;
    }

    const int ns = (int)sys.size();
    n_atoms_off.assign(ns + 1, 0);
    for (int s = 0; s < ns; ++s) {
        const SystemHost& S = sys[s];
        if (S.n <= 0) throw ApiError{LIMA_ERR_STATE, "system " + std::to_string(s) + " has no atoms"};
        for (int d = 0; d < 3; ++d)
            if (!(S.box[d] > 2.0 * rlist))
                throw ApiError{LIMA_ERR_INVALID_ARG, "box edge must exceed 2*(cutoff+skin) in system " + std::to_string(s)};
        if (S.pos.size() != (size_t)3 * S.n) throw ApiError{LIMA_ERR_STATE, "positions not set"};
        n_atoms_off[s + 1] = n_atoms_off[s] + S.n;
    }
    const int N = n_atoms_off[ns];

    // ---- per-system layout
    std::vector<SysDesc> sd(ns);
    std::vector<int> cluster_sys, col_sys;
    int col_off = 0, cl_off = 0, pme_off = 0, pme_coff = 0;
    int col_cap = 64;
    double max_density = 0.0;
    pme_on = false;
    bool has_field = false;
    self_energy.assign(ns, 0.0);
    for (int s = 0; s < ns; ++s) {
        const SystemHost& S = sys[s];
        SysDesc& D = sd[s];
        std::memset(&D, 0, sizeof(D));
        const double V = S.box[0] * S.box[1] * S.box[2];
        const double rho = S.n / V;
        max_density = std::max(max_density, rho);
        const double a = std::cbrt(CLUSTER / rho);
        for (int d = 0; d < 3; ++d) {
            D.box[d] = S.box[d];
            D.inv_box[d] = 1.0 / S.box[d];
            D.boxf[d] = (float)S.box[d];
            D.inv_boxf[d] = (float)(1.0 / S.box[d]);
        }
        for (int d = 0; d < 3; ++d) D.efield[d] = (float)(S.efield[d] * 1000.0);
        if (S.efield[0] != 0.0 || S.efield[1] != 0.0 || S.efield[2] != 0.0) has_field = true;
        D.ncol_x = std::max(1, (int)std::floor(S.box[0] / a));
        D.ncol_y = std::max(1, (int)std::floor(S.box[1] / a));
        D.col_w[0] = (float)(S.box[0] / D.ncol_x);
        D.col_w[1] = (float)(S.box[1] / D.ncol_y);
        D.col_off = col_off;
        const int ncols = D.ncol_x * D.ncol_y;
        const double per_col = (double)S.n / ncols;
        col_cap = std::max(col_cap, (int)std::ceil(3.0 * per_col + 64.0));
        // an inhomogeneous system (a droplet, a slab with vacuum) fills some
        // columns far above the average: size the capacity from the columns the
        // current positions fill (the device binning maps the same way)
        {
            std::vector<int> cc(ncols, 0);
            for (int a = 0; a < S.n; ++a) {
                int c[2];
                const int nc[2] = {D.ncol_x, D.ncol_y};
                for (int d = 0; d < 2; ++d) {
                    const double L = S.box[d];
                    double x = S.pos[3 * (size_t)a + d];
                    if (p.periodic) {
                        x -= L * std::floor(x / L);
                        if (!(x < L)) x -= L;
                        if (!(x >= 0.0)) x = 0.0;
                    }
                    c[d] = (int)std::fmin(std::fmax(x * nc[d] / L, 0.0), (double)(nc[d] - 1));
                }
                ++cc[c[0] + D.ncol_x * c[1]];
            }
            const int fullest = *std::max_element(cc.begin(), cc.end());
            col_cap = std::max(col_cap, (int)std::ceil(1.5 * fullest + 64.0));
        }
        D.atom_off = n_atoms_off[s];
        D.n_atoms = S.n;
        D.max_clusters = (S.n + CLUSTER - 1) / CLUSTER + ncols;
        D.cluster_cap_off = cl_off;
        // pair-kernel warps per i-cluster: one warp per cluster leaves a small
        // system's SMs short of warps (3,000 atoms: 375 warps on 148 SMs), so an
        // engine of one system splits its rows over up to 8 warps, aiming at
        // ~4,096 warps; a batch has warps enough and does not split unless asked
        // (a fixed pair_split applies to every system alike, so a system then
        // gives the same bits alone and in a batch)
        if (p.pair_split > 0) {
            int k = 1;
            while (k * 2 <= std::min(8, p.pair_split)) k *= 2;
            D.nb_parts = k;
        } else if (p.pair_split < 0 && ns == 1) {
            const double ncl = std::max(1.0, std::ceil(S.n / (double)CLUSTER));
            const int e2 = (int)std::floor(std::log2(4096.0 / ncl));
            D.nb_parts = 1 << std::min(3, std::max(0, e2));
        } else {
            D.nb_parts = 1;
        }
        for (int c = 0; c < D.max_clusters; ++c) cluster_sys.push_back(s);
        for (int c = 0; c < ncols; ++c) col_sys.push_back(s);
        col_off += ncols;
        cl_off += D.max_clusters;
        // PME grid
        int g[3] = {0, 0, 0};
        if (p.electrostatics == LIMA_ES_EWALD) {
            if (S.pme_set) {
                for (int d = 0; d < 3; ++d) g[d] = S.pme[d];
            } else if (p.pme_grid[0] > 0) {
                for (int d = 0; d < 3; ++d) g[d] = p.pme_grid[d];
            } else if (p.pme_spacing > 0.0) {
                for (int d = 0; d < 3; ++d) g[d] = fft_friendly((int)std::ceil(S.box[d] / p.pme_spacing));
            }
        }
        if (g[0] > 0) {
            pme_on = true;
            for (int d = 0; d < 3; ++d) {
                if (g[d] < 8) throw ApiError{LIMA_ERR_INVALID_ARG, "PME grid dimension must be >= 8"};
                D.pme_n[d] = g[d];
                D.pme_inv_h[d] = (float)(g[d] / S.box[d]);
            }
            D.pme_off = pme_off;
            D.pme_coff = pme_coff;
            pme_off += g[0] * g[1] * g[2];
            pme_coff += (g[0] / 2 + 1) * g[1] * g[2];
            double q2 = 0.0;
            int nq = 0;
            for (int i = 0; i < S.n; ++i) {
                q2 += (double)S.q[i] * S.q[i];
                nq += S.q[i] != 0.f;
            }
            const double pic = p.ref_compat ? kPiRef : kPi;
            const double self_total = -kappa / std::sqrt(pic) * q2 * kCoulomb;
            // reference quirk: the total self term is added to every charged
            // atom's potential and halved (PME.cuh:417-420, 610-622)
            self_energy[s] = p.ref_compat ? 0.5 * nq * self_total : self_total;
            D.self_energy = self_energy[s];
            D.n_charged = nq;
            // per-atom shares of the self term (per-particle log)
            D.self_per_charge = p.ref_compat ? 1 : 0;
            D.self_coef = p.ref_compat ? (float)(0.5 * self_total) : (float)(-kappa / std::sqrt(pic) * kCoulomb);
        }
    }
    if (col_cap > 8192) throw ApiError{LIMA_ERR_UNSUPPORTED, "column capacity too large (very tall box)"};
    const int n_clusters = cl_off;

    // ---- per-atom static data (original order), exclusions and molecules
    std::vector<int> atom_sys(N);
    std::vector<float> q(N), inv_mass(N);
    std::vector<float2> ljp(N);
    std::vector<std::vector<int>> ex(N);
    UnionFind uf(N);
    BondedTerms H;
    std::vector<int2> bidx, pidx, xidx;
    std::vector<float2> bpar, ipar, ppar;
    std::vector<int4> aidx, didx, iidx;
    std::vector<float4> apar, dpar;
    auto check_idx = [&](const SystemHost& S, int a) {
        if (a < 0 || a >= S.n) throw ApiError{LIMA_ERR_INVALID_ARG, "bonded term atom index out of range"};
    };
    auto exclude_all = [&](const int* t, int k, int off) {
        for (int x = 0; x < k; ++x)
            for (int y = x + 1; y < k; ++y) {
                const int a = t[x] + off, b = t[y] + off;
                if (a == b) continue;
                ex[a].push_back(b);
                ex[b].push_back(a);
            }
    };
    for (int s = 0; s < ns; ++s) {
        const SystemHost& S = sys[s];
        const int off = n_atoms_off[s];
        for (int i = 0; i < S.n; ++i) {
            atom_sys[off + i] = s;
            q[off + i] = S.q[i];
            if (!(S.m[i] > 0.f)) throw ApiError{LIMA_ERR_INVALID_ARG, "atom masses must be > 0"};
            inv_mass[off + i] = 1.f / S.m[i];
            ljp[off + i] = make_float2(0.5f * S.sig[i], std::sqrt(std::max(S.eps[i], 0.f)));
        }
        const bool ex_b = p.exclude_bonded != 0;
        for (size_t t = 0; t < S.bonds.size() / 2; ++t) {
            const int* a = &S.bonds[2 * t];
            check_idx(S, a[0]), check_idx(S, a[1]);
            bidx.push_back(make_int2(a[0] + off, a[1] + off));
            bpar.push_back(make_float2(S.bpar[2 * t], S.bpar[2 * t + 1]));
            uf.unite(a[0] + off, a[1] + off);
            if (ex_b) exclude_all(a, 2, off);
        }
        for (size_t t = 0; t < S.angles.size() / 3; ++t) {
            const int* a = &S.angles[3 * t];
            for (int k = 0; k < 3; ++k) check_idx(S, a[k]);
            aidx.push_back(make_int4(a[0] + off, a[1] + off, a[2] + off, 0));
            apar.push_back(make_float4(S.apar[4 * t], S.apar[4 * t + 1], S.apar[4 * t + 2], S.apar[4 * t + 3]));
            uf.unite(a[0] + off, a[1] + off);
            uf.unite(a[1] + off, a[2] + off);
            if (ex_b) exclude_all(a, 3, off);
        }
        for (size_t t = 0; t < S.dihedrals.size() / 4; ++t) {
            const int* a = &S.dihedrals[4 * t];
            for (int k = 0; k < 4; ++k) check_idx(S, a[k]);
            didx.push_back(make_int4(a[0] + off, a[1] + off, a[2] + off, a[3] + off));
            dpar.push_back(make_float4(S.dpar[3 * t], S.dpar[3 * t + 1], S.dpar[3 * t + 2], 0.f));
            for (int k = 0; k < 3; ++k) uf.unite(a[k] + off, a[k + 1] + off);
            if (ex_b) exclude_all(a, 4, off);
        }
        for (size_t t = 0; t < S.impropers.size() / 4; ++t) {
            const int* a = &S.impropers[4 * t];
            for (int k = 0; k < 4; ++k) check_idx(S, a[k]);
            iidx.push_back(make_int4(a[0] + off, a[1] + off, a[2] + off, a[3] + off));
            ipar.push_back(make_float2(S.ipar[2 * t], S.ipar[2 * t + 1]));
            for (int k = 0; k < 3; ++k) uf.unite(a[k] + off, a[k + 1] + off);
            if (ex_b) exclude_all(a, 4, off);
        }
        for (size_t t = 0; t < S.pairbonds.size() / 2; ++t) {
            const int* a = &S.pairbonds[2 * t];
            check_idx(S, a[0]), check_idx(S, a[1]);
            pidx.push_back(make_int2(a[0] + off, a[1] + off));
            ppar.push_back(make_float2(S.ppar[2 * t], S.ppar[2 * t + 1]));
        }
        for (size_t t = 0; t < S.excl.size() / 2; ++t) {
            const int* a = &S.excl[2 * t];
            check_idx(S, a[0]), check_idx(S, a[1]);
            uf.unite(a[0] + off, a[1] + off);
            exclude_all(a, 2, off);
        }
    }
    // ---- the reference's immediate-neighbour pairs (ref_compat with compounds):
    // every pair inside a compound or across bonded compounds that is not
    // excluded is evaluated with no cutoff by its own kernel, and joins the
    // exclusion lists so that the cutoff pair list skips it
    std::vector<int2> midx;
    if (p.ref_compat) {
        for (int s = 0; s < ns; ++s) {
            const SystemHost& S = sys[s];
            if (S.compound.empty()) continue;
            const int off = n_atoms_off[s];
            std::map<int, std::vector<int>> members;
            for (int i = 0; i < S.n; ++i)
                if (S.compound[i] >= 0) members[S.compound[i]].push_back(i + off);
            auto add_pair = [&](int a, int b) {
                if (a == b) return;
                if (std::find(ex[a].begin(), ex[a].end(), b) != ex[a].end()) return;
                midx.push_back(make_int2(std::min(a, b), std::max(a, b)));
            };
            for (auto& kv : members) {
                const auto& m = kv.second;
                for (size_t x = 0; x < m.size(); ++x)
                    for (size_t y = x + 1; y < m.size(); ++y) add_pair(m[x], m[y]);
            }
            std::set<std::pair<int, int>> seen;
            for (size_t t = 0; t < S.bonded_compounds.size() / 2; ++t) {
                const int c0 = std::min(S.bonded_compounds[2 * t], S.bonded_compounds[2 * t + 1]);
                const int c1 = std::max(S.bonded_compounds[2 * t], S.bonded_compounds[2 * t + 1]);
                if (!seen.insert({c0, c1}).second) continue;
                for (int a : members[c0])
                    for (int b : members[c1]) add_pair(a, b);
            }
        }
        std::sort(midx.begin(), midx.end(), [](int2 u, int2 v) { return u.x != v.x ? u.x < v.x : u.y < v.y; });
        for (const int2 pr : midx) {
            ex[pr.x].push_back(pr.y);
            ex[pr.y].push_back(pr.x);
        }
    }
    std::vector<int> excl_off(N + 1, 0), excl_idx, mol(N);
    for (int a = 0; a < N; ++a) {
        auto& v = ex[a];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        excl_off[a + 1] = excl_off[a] + (int)v.size();
        excl_idx.insert(excl_idx.end(), v.begin(), v.end());
        mol[a] = uf.find(a);
        if (pme_on && !p.ref_compat)
            for (int b : v)
                if (b > a && q[a] != 0.f && q[b] != 0.f) xidx.push_back(make_int2(a, b));
    }

    // ---- pair-list capacity: full neighbour count of clusters times 4 rows per
    // cluster pair (about 5.3 of a pair's 8 j-atoms have an i-atom within the list
    // radius in water, and a cluster's half list is about half its neighbours),
    // with a 1.3x margin
    const double a_cl = std::cbrt(CLUSTER / max_density);
    const double reach = rlist + 1.5 * a_cl;
    const double est = 4.0 / 3.0 * kPi * reach * reach * reach * max_density / CLUSTER;
    // replayed graphs cannot grow the list between rebuilds: give them more room
    int pl_cap = (int)std::ceil((p.use_graphs ? 1.8 : 1.3) * 4.0 * est) + 256;
    pl_cap = (pl_cap + 31) / 32 * 32;
    if (st.pl_cap > pl_cap) pl_cap = st.pl_cap;  // keep a capacity grown earlier

    // ---- device allocation
    // The PME chain and the bonded terms are short, latency-bound kernels; at a
    // higher priority their blocks take SMs as soon as pair-kernel blocks retire
    // instead of queueing behind the whole pair kernel.
    int prio_low = 0, prio_high = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    CK(cudaStreamCreateWithPriority(&s_main, cudaStreamNonBlocking, prio_low));
    CK(cudaStreamCreateWithPriority(&s_bonded, cudaStreamNonBlocking, prio_high));
    CK(cudaStreamCreateWithPriority(&s_pme, cudaStreamNonBlocking, prio_high));
    CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_bonded, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_pme, cudaEventDisableTiming));
    CK(cudaEventCreate(&ev_t0));
    CK(cudaEventCreate(&ev_t1));
    for (auto& pr : ev_ph)
        for (cudaEvent_t& e : pr) CK(cudaEventCreate(&e));

    std::vector<int> nb_warp_off(ns + 1, 0);
    int nb_split = 0;
    for (int s = 0; s < ns; ++s) {
        nb_warp_off[s + 1] = nb_warp_off[s] + sd[s].max_clusters * sd[s].nb_parts;
        if (sd[s].nb_parts > 1) nb_split = 1;
    }

    DevState D{};
    D.n_sys = ns;
    D.nb_warps = nb_warp_off[ns];
    D.nb_split = nb_split;
    D.nb_warp_off = upload(nb_warp_off);
    D.has_field = has_field ? 1 : 0;
    D.periodic = p.periodic ? 1 : 0;
    D.n_atoms = N;
    D.n_clusters = n_clusters;
    D.n_slots = n_clusters * CLUSTER;
    D.n_cols = col_off;
    D.pl_cap = pl_cap;
    D.col_cap = col_cap;
    D.sys = upload(sd);
    D.sys_nclusters = dalloc<int>(ns);
    D.cluster_sys = upload(cluster_sys);
    D.col_sys = upload(col_sys);
    const size_t S = D.n_slots;
    D.px = dalloc<double>(S);
    D.py = dalloc<double>(S);
    D.pz = dalloc<double>(S);
    D.xyzq = dalloc<float4>(S);
    D.ljp = dalloc<float2>(S);
    D.vel = dalloc<float4>(S);
    D.fprev = dalloc<float4>(S);
    D.adam_m = dalloc<float4>(S);
    D.adam_v = dalloc<float4>(S);
    // the three force accumulators in one block, cleared by one memset per step
    D.fx = dalloc<long long>(3 * S);
    D.fy = D.fx + S;
    D.fz = D.fx + 2 * S;
    D.orig = dalloc<int>(S);
    D.slot_mol = dalloc<int>(S);
    D.tvel = dalloc<float4>(S);
    D.tfprev = dalloc<float4>(S);
    D.tadam_m = dalloc<float4>(S);
    D.tadam_v = dalloc<float4>(S);
    D.atom_sys = upload(atom_sys);
    D.slot_of = dalloc<int>(N);
    D.q = upload(q);
    D.inv_mass = upload(inv_mass);
    D.ljp_atom = upload(ljp);
    D.mol = upload(mol);
    D.excl_off = upload(excl_off);
    D.excl_idx = upload(excl_idx);
    D.in_pos = dalloc<double>(3 * (size_t)N);
    D.in_vel = dalloc<float>(3 * (size_t)N);
    D.col_of_atom = dalloc<int>(N);
    D.z_of_atom = dalloc<float>(N);
    D.col_count = dalloc<int>(col_off);
    D.col_fill = dalloc<int>(col_off);
    D.col_atom_start = dalloc<int>(col_off);
    D.col_cl_start = dalloc<int>(col_off);
    D.col_ncl = dalloc<int>(col_off);
    D.col_list = dalloc<int>(N);
    D.new_orig = dalloc<int>(S);
    D.bb_lo = dalloc<float4>(n_clusters);
    D.bb_hi = dalloc<float4>(n_clusters);
    D.bb_molsig = dalloc<unsigned long long>(n_clusters);
    D.pl_count = dalloc<int>(n_clusters);
    D.pl_row = dalloc<int2>((size_t)n_clusters * pl_cap);
    if (D.nb_split) {   // the split pair search's per-warp rows (small systems only)
        D.ps_stage = dalloc<int2>((size_t)D.nb_warps * pl_cap);
        D.ps_stage_count = dalloc<int>(D.nb_warps);
    }
    // auto: prune every 2 steps for one system of at least 1,024 clusters.  A
    // smaller system's pair kernel has too few warps to hide the pass's latency
    // (3,000 atoms: 42 -> 47 us per step with pruning), and a batch of small
    // systems gains nothing (32 systems, 280k atoms: 571 -> 578 us); from
    // 2,000 clusters on it pays (16,828 atoms: 80 -> 76 us; 100,200: 1.5 %).
    // Longer intervals are about even on the 100,200-atom box: 182.7, 183.3,
    // 181.7 and 181.1 us per step pruning every 2, 3, 4 and 5 steps (4.55, 4.67,
    // 4.78 and 4.89 M rows walked of 5.52 M built, 31 us per pass)
    const bool prune_auto = p.nstlist >= 4 && D.n_sys == 1 && n_clusters >= 1024;
    prune_every = p.prune_interval < 0 ? (prune_auto ? 2 : 0) : p.prune_interval;
    if (prune_every >= p.nstlist) prune_every = 0;   // the rebuild already cuts at rc + skin
    rin = rc + (rlist - rc) * (double)prune_every / (double)std::max(1, p.nstlist);
    if (prune_every > 0) {
        D.pl_count_in = dalloc<int>(n_clusters);
        D.pl_row_in = dalloc<int2>((size_t)n_clusters * pl_cap);
        D.walk_count = D.pl_count_in;
        D.walk_row = D.pl_row_in;
    } else {
        D.walk_count = D.pl_count;
        D.walk_row = D.pl_row;
    }
    D.nb_counter = dalloc<int>(1);
    D.status = dalloc<unsigned>(2);   // [0] ST_* flags, [1] largest pair-list row count a search needed
    D.energy = dalloc<long long>((size_t)ns * E_COUNT);
    D.epot = dalloc<long long>(S);
    D.xyz_ref = dalloc<float4>(S);
    D.vscale = upload(std::vector<float>(ns, (float)p.thermostat_scalar));
    d_therm_ke = dalloc<long long>((size_t)ns * E_COUNT);
    therm_T.assign(ns, 0.0);
    therm_scale.assign(ns, p.thermostat_scalar);
    therm_step = -1;
    if (p.log_interval > 0) {
        const int ring = p.log_ring > 0 ? p.log_ring : 5;
        log_pe = dalloc<float4>((size_t)ring * N);
        log_fs = dalloc<float4>((size_t)ring * N);
        log_fill = 0;
        log_ring_steps.clear();
    }

    // ---- PME plan, grids and influence function
    pp = PmePlan{};
    if (pme_on) pp = make_pme(sd, D);
    sd_host = sd;

    // ---- bonded terms
    BondedTerms B{};
    B.nb = (int)bidx.size();
    B.na = (int)aidx.size();
    B.nd = (int)didx.size();
    B.ni = (int)iidx.size();
    B.np = (int)pidx.size();
    B.nx = (int)xidx.size();
    B.nm = (int)midx.size();
    B.midx = upload(midx);
    B.bidx = upload(bidx);
    B.bpar = upload(bpar);
    B.aidx = upload(aidx);
    B.apar = upload(apar);
    B.didx = upload(didx);
    B.dpar = upload(dpar);
    B.iidx = upload(iidx);
    B.ipar = upload(ipar);
    B.pidx = upload(pidx);
    B.ppar = upload(ppar);
    B.xidx = upload(xidx);
    bt = B;
    st = D;

    nb.rc2 = (float)(rc * rc);
    nb.rlist = (float)rlist;
    nb.es_mode = p.electrostatics;
    nb.kappa = (float)kappa;
    nb.ke = (float)kCoulomb;
    nb.two_kappa_sqrtpi = (float)(2.0 * kappa / std::sqrt(p.ref_compat ? kPiRef : kPi));
    nb.mk2_log2e = (float)(-kappa * kappa / std::log(2.0));
    nb.p_kappa = AS_P * (float)kappa;
    nb.em = 0;
    ip.dt = p.dt;
    ip.integrator = p.integrator;
    ip.half_skin2 = (float)(0.25 * (rlist - rc) * (rlist - rc));

    d_disp = dalloc<unsigned>(2);
    d_out_d = dalloc<double>(3 * (size_t)N);
    d_out_f = dalloc<float>(3 * (size_t)N);
    d_maxf = dalloc<float>(1);
    energy_host.assign((size_t)ns * E_COUNT, 0);
    h_pin_bytes = 4 * sizeof(unsigned) + energy_host.size() * sizeof(long long);
    CK(cudaMallocHost((void**)&h_pin, h_pin_bytes));
    std::memset(h_pin, 0, h_pin_bytes);

    built = true;
    state_pending = true;
    energy_valid = false;
}

// Grids, influence function, FFT plans and twiddles of the PME reciprocal part
// for the systems in `sd` (their pme_n set; pme_off/pme_coff are assigned
// here).  Used for the engine's own grid and for the coarse grid of the
// learned correction.
PmePlan lima_engine::make_pme(std::vector<SysDesc>& sd, DevState& D) {
    const int ns = (int)sd.size();
    PmePlan P{};
    int pme_off = 0, pme_coff = 0, max_n = 0;
    for (SysDesc& Dd : sd) {
        if (Dd.pme_n[0] == 0) continue;
        Dd.pme_off = pme_off;
        Dd.pme_coff = pme_coff;
        pme_off += Dd.pme_n[0] * Dd.pme_n[1] * Dd.pme_n[2];
        pme_coff += (Dd.pme_n[0] / 2 + 1) * Dd.pme_n[1] * Dd.pme_n[2];
        for (int d = 0; d < 3; ++d) max_n = std::max(max_n, Dd.pme_n[d]);
    }
    D.pme_total_real = pme_off;
    D.pme_total_cplx = pme_coff;
    D.pme_grid_fx = dalloc<int>(pme_off);
    D.pme_real = dalloc<float>(pme_off);
    D.pme_cplx = dalloc<float2>(pme_coff);
    std::vector<float> theta(pme_coff, 0.f);
    std::vector<char> plans(pme_sys_dev_size() * ns, 0);
    std::vector<int4> ix, iy, iz;
    const int XL = PME_FFT_XLINES, TX = PME_FFT_TX;
    for (int s = 0; s < ns; ++s) {
        const SysDesc& Dd = sd[s];
        if (Dd.pme_n[0] == 0) {
            // a system without a grid still needs a valid (unused) plan
            fill_pme_sys_dev(plans.data() + s * pme_sys_dev_size(), 8, 8, 8);
            continue;
        }
        const int K0 = Dd.pme_n[0], K1 = Dd.pme_n[1], K2 = Dd.pme_n[2], K0h = K0 / 2 + 1;
        if (!fill_pme_sys_dev(plans.data() + s * pme_sys_dev_size(), K0, K1, K2))
            throw ApiError{LIMA_ERR_UNSUPPORTED, "PME grid dimensions must factor into 2, 3, 5 and be <= 256"};
        for (int l = 0; l < K1 * K2; l += XL) ix.push_back(make_int4(s, l, std::min(XL, K1 * K2 - l), 0));
        for (int z = 0; z < K2; ++z)
            for (int x0 = 0; x0 < K0h; x0 += TX) iy.push_back(make_int4(s, x0, z, 0));
        for (int y = 0; y < K1; ++y)
            for (int x0 = 0; x0 < K0h; x0 += TX) iz.push_back(make_int4(s, x0, y, 0));
        const double* L = Dd.box;
        const double V = L[0] * L[1] * L[2];
        const double pic = p.ref_compat ? kPiRef : kPi;
        for (int z = 0; z < K2; ++z)
            for (int y = 0; y < K1; ++y)
                for (int x = 0; x < K0h; ++x) {
                    const int m[3] = {x, y <= K1 / 2 ? y : y - K1, z <= K2 / 2 ? z : z - K2};
                    const int K[3] = {K0, K1, K2};
                    if (m[0] == 0 && m[1] == 0 && m[2] == 0) continue;
                    double kv[3], k2 = 0.0;
                    for (int d = 0; d < 3; ++d) {
                        kv[d] = 2.0 * pic * m[d] / L[d];
                        k2 += kv[d] * kv[d];
                    }
                    double t = kCoulomb * 4.0 * pic / k2 * std::exp(-k2 / (4.0 * kappa * kappa)) / V;
                    if (p.ref_compat) {
                        // PrecomputeGreensFunctionKernel (PME.cuh:434-495): x prod sinc^8
                        double sp = 1.0;
                        for (int d = 0; d < 3; ++d) {
                            const double kh = kv[d] * (L[d] / K[d]) * 0.5;
                            const double sc = std::fabs(kh) < 1e-14 ? 1.0 : std::sin(kh) / kh;
                            sp *= sc * sc * sc * sc;
                        }
                        t *= sp * sp;
                    } else {
                        // SPME: divide by the B-spline modulus of the centred order-4 weights
                        double B = 1.0;
                        for (int d = 0; d < 3; ++d) {
                            const double b = 2.0 / 3.0 + std::cos(2.0 * kPi * m[d] / K[d]) / 3.0;
                            B *= b * b;
                        }
                        t /= B;
                    }
                    theta[Dd.pme_coff + x + (size_t)K0h * (y + (size_t)K1 * z)] = (float)t;
                }
    }
    D.pme_theta = upload(theta);
    // twiddle tables, one per distinct grid length, in FP64 rounded to float
    std::vector<float2> tw;
    std::vector<std::pair<int, int>> tw_offsets;  // (length, offset)
    auto tw_of = [&](int len) {
        for (auto& pr : tw_offsets)
            if (pr.first == len) return pr.second;
        const int off = (int)tw.size();
        for (int k = 0; k < len; ++k) {
            const double a = 2.0 * kPi * k / len;
            tw.push_back(make_float2((float)std::cos(a), (float)-std::sin(a)));
        }
        tw_offsets.push_back({len, off});
        return off;
    };
    for (int s = 0; s < ns; ++s) {
        const int* g = sd[s].pme_n;
        if (g[0] == 0) continue;
        set_pme_sys_twiddles(plans.data() + s * pme_sys_dev_size(), tw_of(g[0]), tw_of(g[1]), tw_of(g[2]));
    }
    D.pme_tw = upload(tw);
    char* dplans = dalloc<char>(plans.size());
    CK(cudaMemcpy(dplans, plans.data(), plans.size(), cudaMemcpyHostToDevice));
    P.sys_plans = dplans;
    P.items_x = upload(ix);
    P.items_y = upload(iy);
    P.items_z = upload(iz);
    P.n_items_x = (int)ix.size();
    P.n_items_y = (int)iy.size();
    P.n_items_z = (int)iz.size();
    P.ref_gather = p.ref_compat ? 1 : 0;
    P.max_n = max_n;
    // plane-fused x+y passes when every system's planes fit in shared memory
    int xy_buf = 0;
    bool xy_ok = true;
    std::vector<int4> ixy;
    for (int s = 0; s < ns; ++s) {
        const int* g = sd[s].pme_n;
        if (g[0] == 0) continue;
        const int b = pme_xy_buffer(g[0], g[1]);
        if (b == 0) xy_ok = false;
        xy_buf = std::max(xy_buf, b);
        for (int z = 0; z < g[2]; ++z) ixy.push_back(make_int4(s, z, 0, 0));
    }
    if (xy_ok && !ixy.empty()) {
        P.items_xy = upload(ixy);
        P.n_items_xy = (int)ixy.size();
        P.xy_buf = xy_buf;
    }
    // spreading and gathering by blocks of columns: the whole z range per block
    // when its box fits in shared memory, else chunks of z nodes (each chunk's
    // CTA walks the block's atoms and keeps the planes it owns)
    std::vector<int4> isp, geo(ns, make_int4(0, 0, 0, 0));
    int box = 0;
    for (int s = 0; s < ns; ++s) {
        const SysDesc& Dd = sd[s];
        if (Dd.pme_n[0] == 0) continue;
        const int NX = pme_spread_box_side(Dd.col_w[0], Dd.pme_inv_h[0]);
        const int NY = pme_spread_box_side(Dd.col_w[1], Dd.pme_inv_h[1]);
        const int ZC = std::min(Dd.pme_n[2], PME_SPREAD_MAX_BOX / (NX * NY));
        if (ZC < 4) {  // a box would not fit: keep per-weight atomics for every system
            isp.clear();
            break;
        }
        geo[s] = make_int4(NX, NY, ZC, 0);
        box = std::max(box, NX * NY * ZC);
        for (int z0 = 0; z0 < Dd.pme_n[2]; z0 += ZC)
            for (int cy = 0; cy < Dd.ncol_y; cy += PME_SPREAD_COLS)
                for (int cx = 0; cx < Dd.ncol_x; cx += PME_SPREAD_COLS) isp.push_back(make_int4(s, cx, cy, z0));
    }
    if (!isp.empty()) {
        P.items_spread = upload(isp);
        P.spread_geo = upload(geo);
        P.n_items_spread = (int)isp.size();
        P.spread_box = box;
    }
    pme_set_smem_limits(max_n, P.n_items_xy > 0 ? xy_buf : 0);
    P.n_sys = ns;
    if (ns > 0) P.sys0 = sd[0];
    return P;
}

// ------------------------------------------------------------ learned PME
// Allocates the coarse-grid view, the feature/target buffers, a dataset ring
// of max_frames frames and the network (Glorot-uniform weights, fixed seed).
void lima_engine::learned_setup(int cx, int cy, int cz, int max_frames) {
    const int ns = (int)sd_host.size();
    for (int s = 0; s < ns; ++s)
        for (int d = 0; d < 3; ++d)
            if (!(sd_host[s].box[d] > 2.0 * (DESC_CUT + 0.1)))
                throw ApiError{LIMA_ERR_INVALID_ARG, "box edge must exceed 1.8 nm for the learned descriptor"};
    const size_t S = st.n_slots;
    // coarse view: same atoms and clusters, own grids, forces into lp_fc
    std::vector<SysDesc> sdc = sd_host;
    for (SysDesc& D : sdc) {
        const int g[3] = {cx, cy, cz};
        for (int d = 0; d < 3; ++d) {
            D.pme_n[d] = g[d];
            D.pme_inv_h[d] = (float)(g[d] / D.box[d]);
        }
    }
    DevState Dc = st;
    pp_c = make_pme(sdc, Dc);
    Dc.sys = upload(sdc);
    lp_fc = dalloc<long long>(3 * S);
    lp_ff = dalloc<long long>(3 * S);
    lp_energy = dalloc<long long>((size_t)st.n_sys * E_COUNT);
    Dc.fx = lp_fc;
    Dc.fy = lp_fc + S;
    Dc.fz = lp_fc + 2 * S;
    Dc.energy = lp_energy;
    st_c = Dc;
    DevState Df = st;
    Df.fx = lp_ff;
    Df.fy = lp_ff + S;
    Df.fz = lp_ff + 2 * S;
    st_f = Df;
    lp_feat = dalloc<float>(S * MLP_IN);
    lp_X = dalloc<__nv_bfloat16>(S * MLP_KIN);
    lp_Y = dalloc<float>(S * 8);
    lp_mean = dalloc<float>(MLP_IN);
    lp_invstd = dalloc<float>(MLP_IN);
    // dataset ring
    ds_cap = max_frames;
    ds_frames = 0;
    ds_feat = dalloc<float>((size_t)max_frames * st.n_atoms * MLP_IN);
    ds_target = dalloc<float>((size_t)max_frames * st.n_atoms * 3);
    // network and training buffers
    MlpModel m{};
    std::mt19937_64 rng(20241203ull);
    for (int l = 0; l < 4; ++l) {
        const int K = MLP_K[l], N = MLP_N[l];
        const int fan_in = l == 0 ? MLP_IN : K, fan_out = l == 3 ? MLP_OUT : N;
        const double a = std::sqrt(6.0 / (fan_in + fan_out)) * (l == 3 ? 0.1 : 1.0);
        std::uniform_real_distribution<double> U(-a, a);
        std::vector<float> w((size_t)K * N, 0.f);
        for (int k = 0; k < fan_in; ++k)
            for (int n = 0; n < fan_out; ++n) w[(size_t)k * N + n] = (float)U(rng);
        m.w[l] = upload(w);
        m.b[l] = dalloc<float>(N);
        m.mw[l] = dalloc<float>((size_t)K * N);
        m.vw[l] = dalloc<float>((size_t)K * N);
        m.mb[l] = dalloc<float>(N);
        m.vb[l] = dalloc<float>(N);
        m.gw[l] = dalloc<float>((size_t)K * N);
        m.gb[l] = dalloc<float>(N);
        m.wb[l] = dalloc<__nv_bfloat16>((size_t)K * (l == 3 ? 16 : N));
        m.wtb[l] = dalloc<__nv_bfloat16>((size_t)N * K);
    }
    const size_t rows_max = std::max<size_t>(S, (size_t)batch_cap);
    m.tmp[0] = dalloc<__nv_bfloat16>(rows_max * MLP_HID);
    m.tmp[1] = dalloc<__nv_bfloat16>(rows_max * MLP_HID);
    const size_t chunks = ((size_t)batch_cap + MLP_CHUNK - 1) / MLP_CHUNK;
    m.part = dalloc<float>(chunks * 128 * 128);
    m.bpart = dalloc<float>(chunks * 128);
    m.max_rows = batch_cap;
    m.tc_err = dalloc<int>(1);
    for (int c = 0; c < MLP_IN; ++c) m.in_mean[c] = 0.f, m.in_std[c] = 1.f;
    mlp = m;
    mlp_sync_bf16(mlp, s_main);
    MlpActs A{};
    for (int l = 0; l < 3; ++l) {
        A.z[l] = dalloc<__nv_bfloat16>((size_t)batch_cap * MLP_HID);
        A.h[l] = dalloc<__nv_bfloat16>((size_t)batch_cap * MLP_HID);
        A.dz[l] = dalloc<__nv_bfloat16>((size_t)batch_cap * MLP_HID);
    }
    A.dz4 = dalloc<__nv_bfloat16>((size_t)batch_cap * 16);
    A.y = dalloc<float>((size_t)batch_cap * 8);
    acts = A;
    batch_X = dalloc<__nv_bfloat16>((size_t)batch_cap * MLP_KIN);
    batch_T = dalloc<float>((size_t)batch_cap * 3);
    batch_raw = dalloc<float>((size_t)batch_cap * MLP_IN);
    d_sums = dalloc<double>(4);
    d_loss = dalloc<double>(1);
    CK(cudaStreamSynchronize(s_main));
    lp_ready = true;
    lp_on = lp_fallback = lp_norm = lp_check_pending = false;
    lp_steps = 0;
    lp_last_rel = -1.0;
}

// coarse-grid reciprocal force into lp_fc, features into lp_feat and, when
// `forward`, the network's prediction into lp_Y
void lima_engine::learned_features(bool forward, cudaStream_t s) {
    CK(cudaMemsetAsync(lp_fc, 0, sizeof(long long) * 3 * (size_t)st.n_slots, s));
    launches += launch_pme(st_c, pp_c, false, s);
    launches += launch_descriptor(st, lp_fc, lp_feat, s);
    if (forward && lp_norm) {
        if (mlp.use_tc) launches += mlp_infer_tc(mlp, st.n_slots, lp_feat, lp_mean, lp_invstd, lp_Y, mlp.tc_err, s);
        else launches += mlp_infer(mlp, st.n_slots, lp_feat, lp_mean, lp_invstd, lp_Y, s);
    }
}

// full-grid reciprocal force into lp_ff (energy, when asked, into the engine's
// own accumulators)
void lima_engine::learned_full(cudaStream_t s, bool energy) {
    CK(cudaMemsetAsync(lp_ff, 0, sizeof(long long) * 3 * (size_t)st.n_slots, s));
    st_f.pme_grid_fx = st.pme_grid_fx;
    st_f.energy = st.energy;
    st_f.atom_energy = st.atom_energy;
    launches += launch_pme(st_f, pp, energy, s);
}

// The reciprocal stage of one step with the correction on.  Every lp_check
// steps (and whenever energies are wanted) the full grid runs as well: its
// forces are the ones applied and the prediction's error against them is
// summed for the host-side check after the step.
void lima_engine::learned_pme_stage(bool energy, cudaStream_t s) {
    const bool check = energy || lp_steps % lp_check == 0;
    learned_features(true, s);
    if (check) {
        learned_full(s, energy);
        CK(cudaMemsetAsync(d_sums, 0, 4 * sizeof(double), s));
        launches += launch_pred_error(st, lp_fc, lp_Y, mlp.out_scale, lp_ff, d_sums, s);
        launches += launch_add_forces(st, lp_ff, s);
        lp_check_pending = true;
    } else {
        launches += launch_mlp_apply(st, lp_fc, lp_Y, mlp.out_scale, s);
    }
    ++lp_steps;
}

void lima_engine::ensure_list() {
    if (state_pending) {
        rebuild(true);
        state_pending = false;
    } else if (list_age >= p.nstlist) {
        rebuild(false);
    }
}

// List rebuild, part one: new slot order and cluster boxes (stages 1-7), no
// host synchronisation.
void lima_engine::start_rebuild(bool from_input) {
    if (from_input) {
        std::vector<double> pos((size_t)3 * st.n_atoms);
        std::vector<float> vel((size_t)3 * st.n_atoms, 0.f);
        for (size_t s = 0; s < sys.size(); ++s) {
            std::copy(sys[s].pos.begin(), sys[s].pos.end(), pos.begin() + 3 * (size_t)n_atoms_off[s]);
            if (sys[s].vel.size() == (size_t)3 * sys[s].n)
                std::copy(sys[s].vel.begin(), sys[s].vel.end(), vel.begin() + 3 * (size_t)n_atoms_off[s]);
        }
        CK(cudaMemcpyAsync(st.in_pos, pos.data(), pos.size() * sizeof(double), cudaMemcpyHostToDevice, s_main));
        CK(cudaMemcpyAsync(st.in_vel, vel.data(), vel.size() * sizeof(float), cudaMemcpyHostToDevice, s_main));
    }
    CK(cudaMemsetAsync(st.status, 0, 2 * sizeof(unsigned), s_main));
    mark(0, 0, s_main);
    launches += launch_rebuild_slots(st, from_input, s_main);
}

// Part two: the pair search, then the host checks the status word.  A column
// overflow rejects the build; a full pair list grows to the largest row count
// the search needed (it counts past the capacity) and only the search is redone
// (the slots are final, and other streams may already be reading them).
void lima_engine::finish_rebuild() {
    for (int attempt = 0; attempt < 3; ++attempt) {
        launches += launch_pairsearch(st, (float)rlist, s_main);
        if (attempt == 0) {
            mark(0, 1, s_main);
            ++rebuilds;
        }
        CK(cudaGetLastError());
        unsigned status[2] = {0u, 0u};
        CK(cudaMemcpyAsync(status, st.status, sizeof(status), cudaMemcpyDeviceToHost, s_main));
        CK(cudaStreamSynchronize(s_main));
        if (status[0] & ST_COLUMN_OVERFLOW) throw ApiError{LIMA_ERR_OVERFLOW, "column capacity exceeded (atoms too dense)"};
        if (!(status[0] & ST_PAIRLIST_OVERFLOW)) {
            list_age = 0;
            return;
        }
        // room for the largest row count of this build plus an eighth for the
        // motion until the next one
        const long long need = (long long)status[1] + status[1] / 8 + 32;
        const long long grown = std::max<long long>((long long)st.pl_cap * 3 / 2, need);
        if (grown > INT_MAX / 2) throw ApiError{LIMA_ERR_OVERFLOW, "pair list too long for one cluster"};
        const int cap = (int)((grown + 31) / 32 * 32);
        for (void* a : {(void*)st.pl_row, (void*)st.pl_row_in, (void*)st.ps_stage}) {
            if (!a) continue;
            cudaFree(a);
            allocs.erase(std::remove(allocs.begin(), allocs.end(), a), allocs.end());
        }
        st.pl_cap = cap;
        st.pl_row = dalloc<int2>((size_t)st.n_clusters * cap);
        if (st.nb_split) st.ps_stage = dalloc<int2>((size_t)st.nb_warps * cap);
        if (prune_every > 0) {
            st.pl_row_in = dalloc<int2>((size_t)st.n_clusters * cap);
            st.walk_row = st.pl_row_in;
        } else {
            st.walk_row = st.pl_row;
        }
        drop_graph();
        CK(cudaMemsetAsync(st.status, 0, 2 * sizeof(unsigned), s_main));
    }
    throw ApiError{LIMA_ERR_OVERFLOW, "pair list overflow persists"};
}

void lima_engine::rebuild(bool from_input) {
    start_rebuild(from_input);
    finish_rebuild();
    // the walked list must follow the new build at once (a pair-list query may
    // come before the next forces)
    if (prune_every > 0) launches += launch_prune(st, (float)rin, s_main);
}

// The list step of forces(): when a rebuild is due, only its first part runs
// here; forces() finishes it after the bonded and PME work has been queued on
// its own streams, so that those overlap the pair search.  Returns whether a
// pair search is pending.
bool lima_engine::begin_list() {
    if (phase_timing) {
        ensure_list();
        return false;
    }
    if (state_pending) {
        start_rebuild(true);
        state_pending = false;
        return true;
    }
    if (list_age >= p.nstlist) {
        start_rebuild(false);
        return true;
    }
    return false;
}

// Pair-list rebuild without the host-side overflow check (inside a CUDA graph);
// the status word is read after the replay.
void lima_engine::rebuild_async() {
    launches += launch_rebuild_slots(st, false, s_main);
    ++rebuilds;
}

// Records use_graphs pair-list periods — each a rebuild, then nstlist steps of
// forces and integration without energies — as one CUDA graph on the main
// stream (the bonded and PME streams join through the fork/join events).
void lima_engine::capture_period() {
    drop_graph();
    const int64_t l0 = launches, r0 = rebuilds;
    const bool pt = phase_timing;
    phase_timing = false;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(s_main, cudaStreamCaptureModeThreadLocal));
    for (int period = 0; period < std::max(1, p.use_graphs); ++period) {
        rebuild_async();
        for (int k = 0; k < p.nstlist; ++k) {
            launches += launch_zero_forces(st, s_main);
            CK(cudaEventRecord(ev_fork, s_main));
            CK(cudaStreamWaitEvent(s_bonded, ev_fork, 0));
            CK(cudaStreamWaitEvent(s_pme, ev_fork, 0));
            launches += launch_bonded(st, bt, false, s_bonded);
            if (pme_on) launches += launch_exclusion_correction(st, bt, nb, false, s_bonded);
            launches += launch_immediate_pairs(st, bt, nb, false, s_bonded);
            CK(cudaEventRecord(ev_bonded, s_bonded));
            if (pme_on) launches += launch_pme(st, pp, false, s_pme);
            CK(cudaEventRecord(ev_pme, s_pme));
            // the period's pair search overlaps its first bonded and PME work
            if (k == 0) launches += launch_pairsearch(st, (float)rlist, s_main);
            if (prune_every > 0 && k % prune_every == 0) launches += launch_prune(st, (float)rin, s_main);
            launches += launch_nonbonded(st, nb, false, s_main, nb_shape);
            CK(cudaStreamWaitEvent(s_main, ev_bonded, 0));
            CK(cudaStreamWaitEvent(s_main, ev_pme, 0));
            launches += launch_integrate(st, ip, false, s_main);
        }
    }
    CK(cudaStreamEndCapture(s_main, &graph));
    const cudaError_t e = cudaGraphInstantiate(&graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(e);
    graph_launches_per_replay = launches - l0;
    launches = l0;
    rebuilds = r0;
    phase_timing = pt;
}

// atom_energy: an energy evaluation that also fills the per-atom shares (epot)
// of a log frame
void lima_engine::forces(bool energy, bool atom_energy) {
    const bool search_pending = begin_list();
    st.atom_energy = energy && atom_energy ? 1 : 0;
    if (energy) {
        CK(cudaMemsetAsync(st.energy, 0, sizeof(long long) * E_COUNT * st.n_sys, s_main));
        if (st.atom_energy) CK(cudaMemsetAsync(st.epot, 0, sizeof(long long) * st.n_slots, s_main));
    }
    launches += launch_zero_forces(st, s_main);
    // with phase timing on, every phase runs on the main stream so that each
    // phase's events bracket that phase alone
    cudaStream_t sb = phase_timing ? s_main : s_bonded;
    cudaStream_t sp = phase_timing ? s_main : s_pme;
    CK(cudaEventRecord(ev_fork, s_main));
    CK(cudaStreamWaitEvent(sb, ev_fork, 0));
    CK(cudaStreamWaitEvent(sp, ev_fork, 0));
    mark(2, 0, sb);
    launches += launch_bonded(st, bt, energy, sb);
    if (pme_on) launches += launch_exclusion_correction(st, bt, nb, energy, sb);
    launches += launch_immediate_pairs(st, bt, nb, energy, sb);
    mark(2, 1, sb);
    CK(cudaEventRecord(ev_bonded, sb));
    if (pme_on) {
        mark(3, 0, sp);
        if (learned_active()) learned_pme_stage(energy, sp);
        else launches += launch_pme(st, pp, energy, sp);
        mark(3, 1, sp);
    }
    CK(cudaEventRecord(ev_pme, sp));
    if (search_pending) finish_rebuild();
    if (prune_every > 0 && (list_age % prune_every == 0 || prune_pending)) {
        launches += launch_prune(st, (float)rin, s_main);
        prune_pending = false;
    }
    mark(1, 0, s_main);
    launches += launch_nonbonded(st, nb, energy, s_main, nb_shape);
    mark(1, 1, s_main);
    CK(cudaStreamWaitEvent(s_main, ev_bonded, 0));
    CK(cudaStreamWaitEvent(s_main, ev_pme, 0));
    CK(cudaGetLastError());
}

void lima_engine::run_steps(int n) {
    CK(cudaEventRecord(ev_t0, s_main));
    int k = 0;
    if (p.use_graphs && !phase_timing && !state_pending && !learned_active() && p.log_interval <= 0) {
        // blocks of use_graphs whole pair-list periods replay as one graph; the
        // last step stays eager so that it can evaluate energies
        const int periods = std::max(1, p.use_graphs), block = periods * p.nstlist;
        while (n - k > block && list_age >= p.nstlist) {
            if (!graph_exec) capture_period();
            CK(cudaMemsetAsync(st.status, 0, sizeof(unsigned), s_main));
            CK(cudaGraphLaunch(graph_exec, s_main));
            launches += graph_launches_per_replay;
            rebuilds += periods;
            ++graph_replays;
            list_age = p.nstlist;
            k += block;
            const int64_t before = step;
            step += block;
            // a thermostat measurement due inside the replayed period is taken after it
            if (p.thermostat_interval > 0 && step / p.thermostat_interval != before / p.thermostat_interval)
                measure_temperature();
        }
    }
    for (; k < n; ++k) {
        const bool log_now = p.log_interval > 0 && step % p.log_interval == 0;
        const bool energy = k == n - 1 || log_now;
        forces(energy, log_now);
        mark(4, 0, s_main);
        launches += launch_integrate(st, ip, energy, s_main);
        mark(4, 1, s_main);
        // logged after the update, as the reference's integration kernel does:
        // new position, this step's potential energy and force, updated speed
        if (log_now) log_frame();
        collect_phases();
        ++list_age;
        ++step;
        if (p.thermostat_interval > 0 && step % p.thermostat_interval == 0) measure_temperature();
        if (lp_check_pending) {
            // full-grid check of the learned correction: fall back to plain
            // PME once the relative reciprocal-force RMSE exceeds the bound
            double sums[4];
            CK(cudaMemcpyAsync(sums, d_sums, sizeof(sums), cudaMemcpyDeviceToHost, s_main));
            CK(cudaStreamSynchronize(s_main));
            lp_check_pending = false;
            lp_last_rel = sums[1] > 0.0 ? std::sqrt(sums[0] / sums[1]) : 0.0;
            if (!(lp_last_rel <= lp_tol)) lp_fallback = true;
        }
    }
    CK(cudaEventRecord(ev_t1, s_main));
    // energies and the status word in one read-back, into pinned memory
    CK(cudaMemcpyAsync(pin_energy(), st.energy, sizeof(long long) * energy_host.size(), cudaMemcpyDeviceToHost,
                       s_main));
    CK(cudaMemcpyAsync(h_pin, st.status, sizeof(unsigned), cudaMemcpyDeviceToHost, s_main));
    CK(cudaStreamSynchronize(s_main));
    CK(cudaGetLastError());
    std::memcpy(energy_host.data(), pin_energy(), sizeof(long long) * energy_host.size());
    last_status = h_pin[0];
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev_t0, ev_t1));
    time_ms += ms;
    timed_steps += n;
    energy_valid = true;
}

// Times `periods` pair-list periods of real MD steps with each launch shape of
// the force-only pair kernel (two rounds, best of each) and keeps the fastest.
// Every shape gives identical results, so the choice changes only the speed.
int lima_engine::autotune(int periods) {
    const int n = std::max(1, periods) * p.nstlist;
    // eight launch shapes of k_nonbonded (0-7), four of the staged kernel (8-11)
    constexpr int NS = 12;
    double best[NS];
    for (int shape = 0; shape < NS; ++shape) {   // first use of each shape, untimed
        best[shape] = 1e300;
        nb_shape = shape;
        drop_graph();
        run_steps(p.nstlist);
    }
    for (int round = 0; round < 3; ++round)
        for (int shape = 0; shape < NS; ++shape) {
            nb_shape = shape;
            drop_graph();
            const double t0 = time_ms;
            run_steps(n);
            best[shape] = std::min(best[shape], time_ms - t0);
        }
    int pick = 0;
    for (int shape = 1; shape < NS; ++shape)
        if (best[shape] < best[pick]) pick = shape;
    for (int shape = 0; shape < NS; ++shape) tune_ms[shape] = best[shape] / n;
    nb_shape = pick;
    nb_tuned = true;
    drop_graph();
    return pick;
}

// Temperature of every system from its kinetic energy (3N - 3 degrees of
// freedom, code/LIMA_BASE/include/PhysicsUtils.cuh:32-34) and, with
// apply_thermostat, the new velocity scale clamp(target/T, 1 -+ 0.001/interval)
// (_Thermostat::ComputeThermostatScalar, Thermostat.cuh:55-67; a zero
// temperature counts as 1 K there).
void lima_engine::measure_temperature() {
    const int ns = st.n_sys;
    CK(cudaMemsetAsync(d_therm_ke, 0, sizeof(long long) * E_COUNT * ns, s_main));
    launches += launch_kinetic(st, d_therm_ke, s_main);
    std::vector<long long> ke((size_t)ns * E_COUNT);
    CK(cudaMemcpyAsync(ke.data(), d_therm_ke, ke.size() * sizeof(long long), cudaMemcpyDeviceToHost, s_main));
    CK(cudaStreamSynchronize(s_main));
    const double kb_na = 1.380649e-23 * 6.02214076e23;
    const double max_step = 0.001 / (double)p.thermostat_interval;
    std::vector<float> scale(ns);
    for (int s = 0; s < ns; ++s) {
        const double K = (double)ke[(size_t)s * E_COUNT + E_KINETIC] / ENERGY_SCALE;
        const double dof = 3.0 * sys[s].n - 3.0;
        const double T = dof > 0.0 ? K * 2.0 / dof / kb_na : 0.0;
        therm_T[s] = T;
        const double Tsafe = T == 0.0 ? 1.0 : T;
        const double target = p.target_temperature > 0.0 ? p.target_temperature : 310.0;
        const double sc = std::min(std::max(target / Tsafe, 1.0 - max_step), 1.0 + max_step);
        if (p.apply_thermostat) therm_scale[s] = sc;
        scale[s] = (float)therm_scale[s];
    }
    therm_step = step;
    if (p.apply_thermostat)
        CK(cudaMemcpyAsync(st.vscale, scale.data(), ns * sizeof(float), cudaMemcpyHostToDevice, s_main));
    CK(cudaStreamSynchronize(s_main));
}

// one frame into the device ring; a full ring goes to host memory
void lima_engine::log_frame() {
    const int ring = p.log_ring > 0 ? p.log_ring : 5;
    const size_t N = st.n_atoms;
    launches += launch_log_frame(st, log_pe + (size_t)log_fill * N, log_fs + (size_t)log_fill * N, s_main);
    log_ring_steps.push_back(step);
    if (++log_fill == ring) flush_log();
}

void lima_engine::flush_log() {
    if (log_fill == 0) return;
    const size_t N = st.n_atoms, n = (size_t)log_fill * N;
    const size_t old = log_host_pe.size();
    log_host_pe.resize(old + n);
    log_host_fs.resize(old + n);
    CK(cudaMemcpyAsync(log_host_pe.data() + old, log_pe, n * sizeof(float4), cudaMemcpyDeviceToHost, s_main));
    CK(cudaMemcpyAsync(log_host_fs.data() + old, log_fs, n * sizeof(float4), cudaMemcpyDeviceToHost, s_main));
    CK(cudaStreamSynchronize(s_main));
    log_host_steps.insert(log_host_steps.end(), log_ring_steps.begin(), log_ring_steps.end());
    log_ring_steps.clear();
    log_fill = 0;
}

void lima_engine::read_energies(lima_energies* e) {
    std::memset(e, 0, sizeof(*e));
    const long long* E = energy_host.data() + (size_t)cur * E_COUNT;
    auto g = [&](int t) { return (double)E[t] / ENERGY_SCALE; };
    e->lj = g(E_LJ);
    e->coulomb_real = g(E_COUL);
    e->pme_recip = g(E_RECIP);
    e->pme_self = pme_on ? self_energy[cur] : 0.0;
    e->pme_excl = g(E_EXCL);
    e->bond = g(E_BOND);
    e->angle = g(E_ANGLE);
    e->dihedral = g(E_DIHEDRAL);
    e->improper = g(E_IMPROPER);
    e->pairbond = g(E_PAIRBOND);
    e->kinetic = g(E_KINETIC);
    e->virial = g(E_VIRIAL);
    e->potential = e->lj + e->coulomb_real + e->pme_recip + e->pme_self + e->pme_excl + e->bond + e->angle +
                   e->dihedral + e->improper + e->pairbond;
    e->total = e->potential + e->kinetic;
    const double kb = 1.380649e-23 * 6.02214076e23;
    const int n = sys[cur].n;
    e->temperature = n > 1 ? 2.0 * e->kinetic / ((3.0 * n - 3.0) * kb) : 0.0;
    e->step = step;
}

// =========================================================================== C-ABI
extern "C" {

void lima_default_params(lima_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->device = 0;
    p->dt = 1e-6;  // 1 fs in ns
    p->cutoff = 1.2;
    p->skin = -1.0;
    p->nstlist = 10;
    p->electrostatics = LIMA_ES_EWALD;
    p->ewald_tol = 1e-5;
    p->integrator = LIMA_INTEGRATOR_LEAPFROG;
    p->thermostat_scalar = 1.0;
    p->exclude_bonded = 1;
    p->use_graphs = 0;
    p->apply_thermostat = 0;
    p->thermostat_interval = 200;   // SimParams::steps_per_temperature_measurement
    p->target_temperature = 310.0;  // Thermostat.cuh:56
    p->log_interval = 0;
    p->log_ring = 5;                // DatabuffersDeviceController::nStepsInBuffer
    p->periodic = 1;                // BoundaryConditionSelect::PBC
    p->prune_interval = -1;         // auto: every 2 steps for one system of >= 1,024 clusters
    p->pair_split = -1;             // auto: split a small single system's pair-kernel rows
}

const char* lima_error_string(int code) {
    switch (code) {
        case LIMA_OK: return "ok";
        case LIMA_ERR_INVALID_ARG: return "invalid argument";
        case LIMA_ERR_CUDA: return "CUDA error";
        case LIMA_ERR_STATE: return "invalid call order";
        case LIMA_ERR_OVERFLOW: return "device list overflow";
        case LIMA_ERR_TIMEOUT: return "device wait timed out";
        case LIMA_ERR_NO_DEVICE: return "no suitable CUDA device";
        case LIMA_ERR_NOT_FINITE: return "non-finite values";
        case LIMA_ERR_UNSUPPORTED: return "unsupported option";
        default: return "unknown error";
    }
}

const char* lima_last_error(const lima_engine* h) { return h ? h->err.c_str() : "null handle"; }

int lima_version(void) { return 1; }

int lima_create_batch(const lima_params* p, int n_systems, lima_engine** out) {
    if (!p || !out || n_systems < 1) return LIMA_ERR_INVALID_ARG;
    if (!(p->dt > 0.0) || !(p->cutoff > 0.0) || p->nstlist < 1) return LIMA_ERR_INVALID_ARG;
    if (p->electrostatics < LIMA_ES_NONE || p->electrostatics > LIMA_ES_EWALD) return LIMA_ERR_INVALID_ARG;
    if (p->integrator != LIMA_INTEGRATOR_LEAPFROG && p->integrator != LIMA_INTEGRATOR_VV) return LIMA_ERR_INVALID_ARG;
    if (p->periodic != 0 && p->periodic != 1) return LIMA_ERR_INVALID_ARG;
    if (!p->periodic && p->electrostatics == LIMA_ES_EWALD) return LIMA_ERR_INVALID_ARG;   // Ewald needs images
    lima_engine* h = new (std::nothrow) lima_engine();
    if (!h) return LIMA_ERR_INVALID_ARG;
    h->p = *p;
    h->sys.resize(n_systems);
    *out = h;
    return LIMA_OK;
}

int lima_create(const lima_params* p, lima_engine** out) { return lima_create_batch(p, 1, out); }

int lima_destroy(lima_engine* h) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (h->device_ok) cudaSetDevice(h->p.device);
    delete h;
    return LIMA_OK;
}

int lima_select_system(lima_engine* h, int system) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (system < 0 || system >= (int)h->sys.size()) return fail(h, LIMA_ERR_INVALID_ARG, "system index out of range");
    h->cur = system;
    return LIMA_OK;
}

int lima_num_systems(const lima_engine* h, int* n) {
    if (!h || !n) return LIMA_ERR_INVALID_ARG;
    *n = (int)h->sys.size();
    return LIMA_OK;
}

// the device state is the current one while the engine is built: copy it back
// into the host-side systems before a topology change drops the device buffers
static void pull_device_state(lima_engine* h) {
    if (!h->built || h->state_pending) return;
    std::vector<double> pp((size_t)3 * h->st.n_atoms);
    std::vector<float> vv((size_t)3 * h->st.n_atoms);
    launch_gather_state(h->st, h->d_out_d, h->d_out_f, h->s_main);
    CK(cudaMemcpyAsync(pp.data(), h->d_out_d, pp.size() * 8, cudaMemcpyDeviceToHost, h->s_main));
    CK(cudaMemcpyAsync(vv.data(), h->d_out_f, vv.size() * 4, cudaMemcpyDeviceToHost, h->s_main));
    CK(cudaStreamSynchronize(h->s_main));
    for (size_t s = 0; s < h->sys.size(); ++s) {
        const size_t o = 3 * (size_t)h->n_atoms_off[s];
        h->sys[s].pos.assign(pp.begin() + o, pp.begin() + o + 3 * h->sys[s].n);
        h->sys[s].vel.assign(vv.begin() + o, vv.begin() + o + 3 * h->sys[s].n);
    }
}

static int topology_changed(lima_engine* h) {
    if (h->device_ok) cudaSetDevice(h->p.device);
    if (h->built) {
        // keep the current state; the topology call itself reports no CUDA error
        try {
            pull_device_state(h);
        } catch (const CudaError&) {
        }
        h->release();
    }
    h->built = false;
    return LIMA_OK;
}

int lima_set_box(lima_engine* h, double lx, double ly, double lz) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (!(lx > 0 && ly > 0 && lz > 0)) return fail(h, LIMA_ERR_INVALID_ARG, "box edges must be > 0");
    SystemHost& S = h->sys[h->cur];
    S.box[0] = lx;
    S.box[1] = ly;
    S.box[2] = lz;
    return topology_changed(h);
}

int lima_set_atoms(lima_engine* h, int n, const float* charge, const float* mass, const float* sigma,
                   const float* epsilon) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (n <= 0 || !charge || !mass || !sigma || !epsilon) return fail(h, LIMA_ERR_INVALID_ARG, "bad atom arrays");
    SystemHost& S = h->sys[h->cur];
    S.n = n;
    S.q.assign(charge, charge + n);
    S.m.assign(mass, mass + n);
    S.sig.assign(sigma, sigma + n);
    S.eps.assign(epsilon, epsilon + n);
    return topology_changed(h);
}

static int set_terms(lima_engine* h, int n, const int32_t* atoms, int k, const float* par, int np,
                     std::vector<int32_t>& dst_i, std::vector<float>& dst_p) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (n < 0 || (n > 0 && (!atoms || (np > 0 && !par)))) return fail(h, LIMA_ERR_INVALID_ARG, "bad term arrays");
    dst_i.assign(atoms, atoms + (size_t)n * k);
    if (np > 0) dst_p.assign(par, par + (size_t)n * np);
    return topology_changed(h);
}

int lima_set_bonds(lima_engine* h, int n, const int32_t* a, const float* p) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return set_terms(h, n, a, 2, p, 2, h->sys[h->cur].bonds, h->sys[h->cur].bpar);
}
int lima_set_angles(lima_engine* h, int n, const int32_t* a, const float* p) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return set_terms(h, n, a, 3, p, 4, h->sys[h->cur].angles, h->sys[h->cur].apar);
}
int lima_set_dihedrals(lima_engine* h, int n, const int32_t* a, const float* p) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return set_terms(h, n, a, 4, p, 3, h->sys[h->cur].dihedrals, h->sys[h->cur].dpar);
}
int lima_set_impropers(lima_engine* h, int n, const int32_t* a, const float* p) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return set_terms(h, n, a, 4, p, 2, h->sys[h->cur].impropers, h->sys[h->cur].ipar);
}
int lima_set_pairbonds(lima_engine* h, int n, const int32_t* a, const float* p) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return set_terms(h, n, a, 2, p, 2, h->sys[h->cur].pairbonds, h->sys[h->cur].ppar);
}
int lima_set_exclusions(lima_engine* h, int n, const int32_t* a) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    std::vector<float> unused;
    return set_terms(h, n, a, 2, nullptr, 0, h->sys[h->cur].excl, unused);
}

int lima_set_compounds(lima_engine* h, int n_atoms, const int32_t* compound, int n_bonded, const int32_t* bonded) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    SystemHost& S = h->sys[h->cur];
    if (n_atoms != S.n || (n_atoms > 0 && !compound) || n_bonded < 0 || (n_bonded > 0 && !bonded))
        return fail(h, LIMA_ERR_INVALID_ARG, "compound arrays must cover every atom of the system");
    std::vector<int> count(std::max(n_atoms, 1), 0);
    for (int i = 0; i < n_atoms; ++i) {
        const int c = compound[i];
        if (c < -1 || c >= n_atoms) return fail(h, LIMA_ERR_INVALID_ARG, "compound id out of range");
        if (c >= 0 && ++count[c] > 32)
            return fail(h, LIMA_ERR_INVALID_ARG, "a compound holds at most 32 atoms (MAX_COMPOUND_PARTICLES)");
    }
    std::vector<int> nb(std::max(n_atoms, 1), 0);
    for (int t = 0; t < n_bonded; ++t) {
        const int a = bonded[2 * t], b = bonded[2 * t + 1];
        if (a < 0 || b < 0 || a >= n_atoms || b >= n_atoms || a == b || !count[a] || !count[b])
            return fail(h, LIMA_ERR_INVALID_ARG, "bonded compound pair names a missing compound");
        if (++nb[a] > 6 || ++nb[b] > 6)
            return fail(h, LIMA_ERR_INVALID_ARG, "a compound is bonded to at most 6 others (max_bonded_compounds)");
    }
    S.compound.assign(compound, compound + n_atoms);
    S.bonded_compounds.assign(bonded, bonded + 2 * (size_t)n_bonded);
    return topology_changed(h);
}

int lima_set_electric_field(lima_engine* h, double ex, double ey, double ez) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (!(std::isfinite(ex) && std::isfinite(ey) && std::isfinite(ez)))
        return fail(h, LIMA_ERR_INVALID_ARG, "electric field must be finite");
    SystemHost& S = h->sys[h->cur];
    S.efield[0] = ex;
    S.efield[1] = ey;
    S.efield[2] = ez;
    return topology_changed(h);
}

int lima_set_pme_grid(lima_engine* h, int nx, int ny, int nz) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (nx < 0 || ny < 0 || nz < 0) return fail(h, LIMA_ERR_INVALID_ARG, "bad PME grid");
    SystemHost& S = h->sys[h->cur];
    S.pme[0] = nx;
    S.pme[1] = ny;
    S.pme[2] = nz;
    S.pme_set = true;
    return topology_changed(h);
}

int lima_set_state(lima_engine* h, const double* pos, const float* vel) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    SystemHost& S = h->sys[h->cur];
    if (S.n <= 0) return fail(h, LIMA_ERR_STATE, "lima_set_atoms must precede lima_set_state");
    if (!pos) return fail(h, LIMA_ERR_INVALID_ARG, "positions required");
    return guarded(h, [&]() {
        if (h->built && !h->state_pending) {
            // Fast path: the atoms keep their slots; the pair list stays valid while no
            // atom has moved more than half the Verlet buffer since it was built.  The
            // input is staged and checked on the device (finite, largest move) before
            // it replaces the slot state.
            // positions on the main stream, checked as soon as they arrive;
            // velocities (needed only by the commit) on a second stream, so that
            // their copy overlaps the check and its read-back
            cudaStream_t s = h->s_main, sv = h->s_bonded;
            const size_t o = 3 * (size_t)h->n_atoms_off[h->cur];
            CK(cudaMemcpyAsync(h->st.in_pos + o, pos, 3 * (size_t)S.n * sizeof(double), cudaMemcpyHostToDevice, s));
            CK(cudaEventRecord(h->ev_fork, s));
            CK(cudaStreamWaitEvent(sv, h->ev_fork, 0));
            if (vel)
                CK(cudaMemcpyAsync(h->st.in_vel + o, vel, 3 * (size_t)S.n * sizeof(float), cudaMemcpyHostToDevice, sv));
            else
                CK(cudaMemsetAsync(h->st.in_vel + o, 0, 3 * (size_t)S.n * sizeof(float), sv));
            CK(cudaEventRecord(h->ev_bonded, sv));
            CK(cudaMemsetAsync(h->d_disp, 0, 2 * sizeof(unsigned), s));
            h->launches += launch_check_state(h->st, h->n_atoms_off[h->cur], S.n, h->d_disp, s);
            CK(cudaMemcpyAsync(h->h_pin + 2, h->d_disp, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            const unsigned word[2] = {h->h_pin[2], h->h_pin[3]};
            if (word[1] & 1u) {
                CK(cudaStreamSynchronize(sv));   // the caller may reuse its buffers on return
                return fail(h, LIMA_ERR_NOT_FINITE, "non-finite position");
            }
            CK(cudaStreamWaitEvent(s, h->ev_bonded, 0));
            h->launches += launch_load_state(h->st, h->n_atoms_off[h->cur], S.n, s);
            // the caller's velocity buffer is read by the copy: done before return
            CK(cudaStreamSynchronize(sv));
            const unsigned bits = word[0];
            float d2;
            std::memcpy(&d2, &bits, sizeof(float));
            // a moved state must keep every atom within half the Verlet buffer of its
            // build position; one handed back unchanged is the engine's own state and
            // keeps the usual nstlist cadence, as stepping without the hand-in would
            const double half_skin = 0.5 * (h->rlist - h->p.cutoff);
            if ((word[1] & 2u) && !((double)d2 < half_skin * half_skin))
                h->list_age = h->p.nstlist;   // rebuild before the next forces
            // moved atoms: the inner (pruned) list follows the new positions
            if (word[1] & 2u) h->prune_pending = true;
            h->energy_valid = false;
            ++h->state_fast_loads;
            return LIMA_OK;
        }
        for (int i = 0; i < 3 * S.n; ++i)
            if (!std::isfinite(pos[i])) return fail(h, LIMA_ERR_NOT_FINITE, "non-finite position");
        // pull the device state of the other systems first so they are kept
        if (h->built && !h->state_pending && h->sys.size() > 1) {
            std::vector<double> pp((size_t)3 * h->st.n_atoms);
            std::vector<float> vv((size_t)3 * h->st.n_atoms);
            launch_gather_state(h->st, h->d_out_d, h->d_out_f, h->s_main);
            CK(cudaMemcpyAsync(pp.data(), h->d_out_d, pp.size() * 8, cudaMemcpyDeviceToHost, h->s_main));
            CK(cudaMemcpyAsync(vv.data(), h->d_out_f, vv.size() * 4, cudaMemcpyDeviceToHost, h->s_main));
            CK(cudaStreamSynchronize(h->s_main));
            for (size_t s = 0; s < h->sys.size(); ++s) {
                if ((int)s == h->cur) continue;
                const size_t o = 3 * (size_t)h->n_atoms_off[s];
                h->sys[s].pos.assign(pp.begin() + o, pp.begin() + o + 3 * h->sys[s].n);
                h->sys[s].vel.assign(vv.begin() + o, vv.begin() + o + 3 * h->sys[s].n);
            }
        }
        S.pos.assign(pos, pos + 3 * (size_t)S.n);
        if (vel) S.vel.assign(vel, vel + 3 * (size_t)S.n);
        else S.vel.assign(3 * (size_t)S.n, 0.f);
        h->state_pending = true;
        return LIMA_OK;
    });
}

static int ensure_built(lima_engine* h) {
    if (!h->built) h->setup();
    return LIMA_OK;
}

int lima_get_state(lima_engine* h, double* pos, float* vel) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return guarded(h, [&]() {
        const SystemHost& S = h->sys[h->cur];
        if (!h->built || h->state_pending) {
            if (pos) std::copy(S.pos.begin(), S.pos.end(), pos);
            if (vel) {
                if (S.vel.empty()) std::fill(vel, vel + 3 * S.n, 0.f);
                else std::copy(S.vel.begin(), S.vel.end(), vel);
            }
            return LIMA_OK;
        }
        launch_gather_state(h->st, h->d_out_d, h->d_out_f, h->s_main);
        const size_t o = 3 * (size_t)h->n_atoms_off[h->cur];
        if (pos) CK(cudaMemcpyAsync(pos, h->d_out_d + o, 3 * (size_t)S.n * 8, cudaMemcpyDeviceToHost, h->s_main));
        if (vel) CK(cudaMemcpyAsync(vel, h->d_out_f + o, 3 * (size_t)S.n * 4, cudaMemcpyDeviceToHost, h->s_main));
        CK(cudaStreamSynchronize(h->s_main));
        return LIMA_OK;
    });
}

int lima_compute_forces(lima_engine* h, int flags) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return guarded(h, [&]() {
        ensure_built(h);
        const bool energy = (flags & LIMA_CALC_ENERGY) != 0;
        h->forces(energy);
        if (energy) {
            CK(cudaMemcpyAsync(h->pin_energy(), h->st.energy, sizeof(long long) * h->energy_host.size(),
                               cudaMemcpyDeviceToHost, h->s_main));
        }
        CK(cudaStreamSynchronize(h->s_main));
        CK(cudaGetLastError());
        if (energy) {
            std::memcpy(h->energy_host.data(), h->pin_energy(), sizeof(long long) * h->energy_host.size());
            h->energy_valid = true;
        }
        return LIMA_OK;
    });
}

int lima_step(lima_engine* h, int n_steps) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (n_steps < 0) return fail(h, LIMA_ERR_INVALID_ARG, "n_steps < 0");
    return guarded(h, [&]() {
        ensure_built(h);
        if (n_steps == 0) return LIMA_OK;
        h->run_steps(n_steps);
        const unsigned status = h->last_status;   // read back with the energies
        if (status & ST_NONFINITE) return fail(h, LIMA_ERR_NOT_FINITE, "non-finite force during stepping");
        if (status & (ST_PAIRLIST_OVERFLOW | ST_COLUMN_OVERFLOW))
            return fail(h, LIMA_ERR_OVERFLOW, "pair list or column capacity exceeded inside a graph replay");
        return LIMA_OK;
    });
}

int lima_minimize(lima_engine* h, double force_tol, int max_steps, int* steps_taken, double* max_force) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (max_steps < 0) return fail(h, LIMA_ERR_INVALID_ARG, "max_steps < 0");
    return guarded(h, [&]() {
        ensure_built(h);
        h->nb.em = 1;
        int k = 0;
        float fmax = 0.f;
        const int check_every = 10;
        for (; k < max_steps; ++k) {
            h->forces(false);
            if (k % check_every == 0 || k == max_steps - 1) {
                CK(cudaMemsetAsync(h->d_maxf, 0, sizeof(float), h->s_main));
                launch_max_force(h->st, h->d_maxf, h->s_main);
                CK(cudaMemcpyAsync(&fmax, h->d_maxf, sizeof(float), cudaMemcpyDeviceToHost, h->s_main));
                CK(cudaStreamSynchronize(h->s_main));
                if (fmax <= force_tol) break;
            }
            launch_em_step(h->st, k + 1, nullptr, h->s_main);
            ++h->list_age;
        }
        CK(cudaStreamSynchronize(h->s_main));
        h->nb.em = 0;
        if (steps_taken) *steps_taken = k;
        if (max_force) *max_force = fmax;
        return LIMA_OK;
    });
}

int lima_get_forces(lima_engine* h, double* forces) {
    if (!h || !forces) return LIMA_ERR_INVALID_ARG;
    if (!h->built || h->state_pending) return fail(h, LIMA_ERR_STATE, "no forces computed yet");
    return guarded(h, [&]() {
        launch_gather_forces(h->st, h->d_out_d, h->s_main);
        const size_t o = 3 * (size_t)h->n_atoms_off[h->cur];
        CK(cudaMemcpyAsync(forces, h->d_out_d + o, 3 * (size_t)h->sys[h->cur].n * 8, cudaMemcpyDeviceToHost, h->s_main));
        CK(cudaStreamSynchronize(h->s_main));
        return LIMA_OK;
    });
}

int lima_get_energies(lima_engine* h, lima_energies* e) {
    if (!h || !e) return LIMA_ERR_INVALID_ARG;
    if (!h->energy_valid) return fail(h, LIMA_ERR_STATE, "no energies evaluated yet");
    h->read_energies(e);
    return LIMA_OK;
}

int lima_get_pairlist(lima_engine* h, int64_t cap, int32_t* pairs, int64_t* n) {
    if (!h || !n || cap < 0 || (cap > 0 && !pairs)) return LIMA_ERR_INVALID_ARG;
    return guarded(h, [&]() {
        ensure_built(h);
        if (h->state_pending) {
            h->rebuild(true);
            h->state_pending = false;
        }
        // count first, then fill
        unsigned long long* dcount = h->dalloc<unsigned long long>(1);
        launch_pairlist_dump(h->st, h->nb, 0, nullptr, dcount, h->s_main);
        unsigned long long total = 0;
        CK(cudaMemcpyAsync(&total, dcount, 8, cudaMemcpyDeviceToHost, h->s_main));
        CK(cudaStreamSynchronize(h->s_main));
        int* dpairs = h->dalloc<int>(2 * std::max<unsigned long long>(total, 1));
        CK(cudaMemsetAsync(dcount, 0, 8, h->s_main));
        launch_pairlist_dump(h->st, h->nb, (long long)total, dpairs, dcount, h->s_main);
        std::vector<int> hp(2 * total);
        if (total) CK(cudaMemcpyAsync(hp.data(), dpairs, hp.size() * 4, cudaMemcpyDeviceToHost, h->s_main));
        CK(cudaStreamSynchronize(h->s_main));
        for (void* a : {(void*)dcount, (void*)dpairs}) {
            cudaFree(a);
            h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), a), h->allocs.end());
        }
        // keep the selected system's pairs, local indices, sorted
        const int off = h->n_atoms_off[h->cur], end = h->n_atoms_off[h->cur + 1];
        std::vector<std::pair<int, int>> v;
        v.reserve(total);
        for (unsigned long long k = 0; k < total; ++k) {
            const int a = hp[2 * k], b = hp[2 * k + 1];
            if (a >= off && a < end) v.emplace_back(a - off, b - off);
        }
        std::sort(v.begin(), v.end());
        *n = (int64_t)v.size();
        for (int64_t k = 0; k < (int64_t)v.size() && k < cap; ++k) {
            pairs[2 * k] = v[k].first;
            pairs[2 * k + 1] = v[k].second;
        }
        return LIMA_OK;
    });
}

int lima_get_pairlist_stats(lima_engine* h, lima_pairlist_stats* out) {
    if (!h || !out) return LIMA_ERR_INVALID_ARG;
    return guarded(h, [&]() {
        ensure_built(h);
        if (h->state_pending) {
            h->rebuild(true);
            h->state_pending = false;
        }
        *out = lima_pairlist_stats{};
        std::vector<int> cnt(h->st.n_clusters), cntw(h->st.n_clusters);
        CK(cudaMemcpyAsync(cnt.data(), h->st.pl_count, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost,
                           h->s_main));
        CK(cudaMemcpyAsync(cntw.data(), h->st.walk_count, cntw.size() * sizeof(int), cudaMemcpyDeviceToHost,
                           h->s_main));
        unsigned long long* dcount = h->dalloc<unsigned long long>(1);
        CK(cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), h->s_main));
        launch_pairlist_dump(h->st, h->nb, 0, nullptr, dcount, h->s_main);
        unsigned long long got[2] = {0, 0};
        CK(cudaMemcpyAsync(got, dcount, 8, cudaMemcpyDeviceToHost, h->s_main));
        CK(cudaStreamSynchronize(h->s_main));
        cudaFree(dcount);
        h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)dcount), h->allocs.end());
        long long rows = 0, walked = 0;
        for (int c : cnt) rows += std::min(c, h->st.pl_cap);
        for (int c : cntw) walked += std::min(c, h->st.pl_cap);
        out->rows_built = rows;
        out->rows_walked = walked;
        out->pairs_evaluated = walked * CLUSTER;
        out->pairs_in_cutoff = (int64_t)got[0];
        return LIMA_OK;
    });
}

int lima_get_status(lima_engine* h, uint32_t* status) {
    if (!h || !status) return LIMA_ERR_INVALID_ARG;
    *status = 0;
    if (!h->built) return LIMA_OK;
    return guarded(h, [&]() {
        unsigned s = 0;
        CK(cudaMemcpy(&s, h->st.status, sizeof(unsigned), cudaMemcpyDeviceToHost));
        *status = s | (h->lp_fallback ? (unsigned)LIMA_STATUS_MLP_FALLBACK : 0u);
        return LIMA_OK;
    });
}

int lima_clear_status(lima_engine* h) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (!h->built) return LIMA_OK;
    return guarded(h, [&]() {
        CK(cudaMemset(h->st.status, 0, sizeof(unsigned)));
        return LIMA_OK;
    });
}

int lima_get_timings(lima_engine* h, lima_timings* t) {
    if (!h || !t) return LIMA_ERR_INVALID_ARG;
    std::memset(t, 0, sizeof(*t));
    const double ns = h->timed_steps ? (double)h->timed_steps : 1.0;
    t->steps = h->timed_steps;
    t->rebuilds = h->rebuilds;
    t->kernel_launches = h->launches;
    t->step = 1000.0 * h->time_ms / ns;
    t->nblist = h->rebuilds ? 1000.0 * h->phase_ms[0] / (double)h->rebuilds : 0.0;
    t->nonbonded = 1000.0 * h->phase_ms[1] / ns;
    t->bonded = 1000.0 * h->phase_ms[2] / ns;
    t->pme = 1000.0 * h->phase_ms[3] / ns;
    t->integrate = 1000.0 * h->phase_ms[4] / ns;
    t->pair_shape = h->nb_shape;
    return LIMA_OK;
}

int lima_reset_timings(lima_engine* h) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    h->time_ms = 0.0;
    h->timed_steps = 0;
    h->rebuilds = 0;
    h->launches = 0;
    for (int k = 0; k < 5; ++k) h->phase_ms[k] = 0.0, h->phase_used[k] = 0;
    return LIMA_OK;
}

int lima_enable_phase_timing(lima_engine* h, int enable) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    h->phase_timing = enable != 0;
    return LIMA_OK;
}

// ------------------------------------------------------------ learned PME
static int learned_ready(lima_engine* h) {
    if (!h->built || !h->lp_ready) return fail(h, LIMA_ERR_STATE, "lima_learned_pme_setup must come first");
    return LIMA_OK;
}

int lima_learned_pme_setup(lima_engine* h, int cx, int cy, int cz, int max_frames) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (cx < 8 || cy < 8 || cz < 8 || max_frames < 1)
        return fail(h, LIMA_ERR_INVALID_ARG, "coarse grid dimensions must be >= 8 and max_frames >= 1");
    return guarded(h, [&]() {
        ensure_built(h);
        if (!h->pme_on) return fail(h, LIMA_ERR_STATE, "the learned correction needs PME electrostatics");
        h->learned_setup(cx, cy, cz, max_frames);
        return LIMA_OK;
    });
}

int lima_learned_pme_collect(lima_engine* h) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return guarded(h, [&]() {
        if (int e = learned_ready(h)) return e;
        h->ensure_list();
        cudaStream_t s = h->s_main;
        h->learned_features(false, s);
        h->learned_full(s, false);
        const int N = h->st.n_atoms;
        const int slot = h->ds_frames % h->ds_cap;
        float* rf = h->ds_feat + (size_t)slot * N * MLP_IN;
        float* rt = h->ds_target + (size_t)slot * N * 3;
        h->launches += launch_collect(h->st, h->lp_feat, h->lp_fc, h->lp_ff, rf, rt, s);
        if (!h->lp_norm) {
            // the first frame fixes the input normalisation and the output scale
            std::vector<float> f((size_t)N * MLP_IN), t((size_t)N * 3);
            CK(cudaMemcpyAsync(f.data(), rf, f.size() * 4, cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(t.data(), rt, t.size() * 4, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            std::vector<float> mean(MLP_IN), inv(MLP_IN);
            for (int c = 0; c < MLP_IN; ++c) {
                double m1 = 0.0, m2 = 0.0;
                for (int a = 0; a < N; ++a) {
                    const double v = f[(size_t)a * MLP_IN + c];
                    m1 += v;
                    m2 += v * v;
                }
                m1 /= N;
                const double sd = std::sqrt(std::max(m2 / N - m1 * m1, 0.0));
                mean[c] = (float)m1;
                h->mlp.in_mean[c] = (float)m1;
                h->mlp.in_std[c] = (float)(sd > 1e-6 ? sd : 1.0);
                inv[c] = 1.f / h->mlp.in_std[c];
            }
            double r2 = 0.0;
            for (float v : t) r2 += (double)v * v;
            const double rms = std::sqrt(r2 / std::max<size_t>(t.size(), 1));
            h->mlp.out_scale = (float)(rms > 0.0 ? rms : 1.0);
            CK(cudaMemcpyAsync(h->lp_mean, mean.data(), MLP_IN * 4, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(h->lp_invstd, inv.data(), MLP_IN * 4, cudaMemcpyHostToDevice, s));
            h->lp_norm = true;
        }
        CK(cudaStreamSynchronize(s));
        ++h->ds_frames;
        return LIMA_OK;
    });
}

int lima_learned_pme_train(lima_engine* h, int epochs, int batch, float lr, uint64_t seed, double* final_loss) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (epochs < 0 || batch < 16 || !(lr >= 0.f)) return fail(h, LIMA_ERR_INVALID_ARG, "bad training arguments");
    return guarded(h, [&]() {
        if (int e = learned_ready(h)) return e;
        if (h->ds_frames == 0) return fail(h, LIMA_ERR_STATE, "no frames collected");
        if (batch > h->batch_cap) return fail(h, LIMA_ERR_INVALID_ARG, "batch larger than 65536 rows");
        cudaStream_t s = h->s_main;
        const size_t rows = (size_t)std::min(h->ds_frames, h->ds_cap) * h->st.n_atoms;
        if (rows > (size_t)INT32_MAX) return fail(h, LIMA_ERR_UNSUPPORTED, "dataset above 2^31 rows");
        if (h->d_idx_cap < rows) {
            if (h->d_idx) {
                cudaFree(h->d_idx);
                h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->d_idx), h->allocs.end());
            }
            h->d_idx = h->dalloc<int>(rows);
            h->d_idx_cap = rows;
        }
        std::vector<int> idx(rows);
        std::iota(idx.begin(), idx.end(), 0);
        const float inv_scale = 1.f / h->mlp.out_scale;
        double last = 0.0;
        for (int ep = 0; ep < epochs; ++ep) {
            std::mt19937_64 rng(seed * 1000003ull + (uint64_t)ep);
            for (size_t i = rows - 1; i > 0; --i) {
                std::uniform_int_distribution<size_t> U(0, i);
                std::swap(idx[i], idx[U(rng)]);
            }
            CK(cudaMemcpyAsync(h->d_idx, idx.data(), rows * sizeof(int), cudaMemcpyHostToDevice, s));
            CK(cudaMemsetAsync(h->d_loss, 0, sizeof(double), s));
            for (size_t off = 0; off < rows; off += batch) {
                const int n = (int)std::min<size_t>(batch, rows - off);
                h->launches += launch_gather_batch(h->ds_feat, h->ds_target, h->d_idx + off, n, h->lp_mean,
                                                   h->lp_invstd, inv_scale, h->batch_X, h->batch_T, s);
                h->launches += mlp_train_step(h->mlp, n, h->batch_X, h->batch_T, h->acts, lr, h->d_loss, s);
            }
            double sum = 0.0;
            CK(cudaMemcpyAsync(&sum, h->d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            last = sum / (3.0 * rows);
        }
        CK(cudaStreamSynchronize(s));
        if (final_loss) *final_loss = last;
        return LIMA_OK;
    });
}

int lima_learned_pme_enable(lima_engine* h, int on, int check_interval, double tolerance) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (int e = learned_ready(h)) return e;
    if (on && !h->lp_norm) return fail(h, LIMA_ERR_STATE, "collect at least one frame before enabling");
    h->lp_on = on != 0;
    h->lp_check = check_interval > 0 ? check_interval : 50;
    h->lp_tol = tolerance > 0.0 ? tolerance : 1e-3;
    h->lp_fallback = false;
    h->lp_check_pending = false;
    h->lp_steps = 0;
    h->lp_last_rel = -1.0;
    return LIMA_OK;
}

int lima_learned_pme_eval(lima_engine* h, double* coarse_rel, double* learned_rel) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    return guarded(h, [&]() {
        if (int e = learned_ready(h)) return e;
        if (!h->lp_norm) return fail(h, LIMA_ERR_STATE, "collect at least one frame first");
        h->ensure_list();
        cudaStream_t s = h->s_main;
        h->learned_features(true, s);
        h->learned_full(s, false);
        CK(cudaMemsetAsync(h->d_sums, 0, 4 * sizeof(double), s));
        h->launches += launch_pred_error(h->st, h->lp_fc, h->lp_Y, h->mlp.out_scale, h->lp_ff, h->d_sums, s);
        double sums[4];
        CK(cudaMemcpyAsync(sums, h->d_sums, sizeof(sums), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const double den = sums[1] > 0.0 ? sums[1] : 1.0;
        if (coarse_rel) *coarse_rel = std::sqrt(sums[2] / den);
        if (learned_rel) *learned_rel = std::sqrt(sums[0] / den);
        return LIMA_OK;
    });
}

int lima_learned_pme_status(lima_engine* h, int* active, int* fell_back, double* last_rel) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (active) *active = h->learned_active() ? 1 : 0;
    if (fell_back) *fell_back = h->lp_fallback ? 1 : 0;
    if (last_rel) *last_rel = h->lp_last_rel;
    return LIMA_OK;
}

int lima_learned_pme_weights(lima_engine* h, int get, float* buf, int64_t n, int64_t* needed) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (needed) *needed = MLP_NSTATE;
    if (!buf) return LIMA_OK;
    if (n < MLP_NSTATE) return fail(h, LIMA_ERR_INVALID_ARG, "weight buffer too small");
    return guarded(h, [&]() {
        if (int e = learned_ready(h)) return e;
        MlpModel& m = h->mlp;
        size_t off = 0;
        for (int l = 0; l < 4; ++l) {
            const size_t nw = (size_t)MLP_K[l] * MLP_N[l], nb = MLP_N[l];
            if (get) {
                CK(cudaMemcpy(buf + off, m.w[l], nw * 4, cudaMemcpyDeviceToHost));
                CK(cudaMemcpy(buf + off + nw, m.b[l], nb * 4, cudaMemcpyDeviceToHost));
            } else {
                CK(cudaMemcpy(m.w[l], buf + off, nw * 4, cudaMemcpyHostToDevice));
                CK(cudaMemcpy(m.b[l], buf + off + nw, nb * 4, cudaMemcpyHostToDevice));
            }
            off += nw + nb;
        }
        if (get) {
            std::copy(m.in_mean, m.in_mean + MLP_IN, buf + off);
            std::copy(m.in_std, m.in_std + MLP_IN, buf + off + MLP_IN);
            buf[off + 2 * MLP_IN] = m.out_scale;
        } else {
            std::vector<float> inv(MLP_IN);
            for (int c = 0; c < MLP_IN; ++c) {
                const float sd = buf[off + MLP_IN + c];
                if (!(sd > 0.f)) return fail(h, LIMA_ERR_INVALID_ARG, "input scales must be > 0");
                m.in_mean[c] = buf[off + c];
                m.in_std[c] = sd;
                inv[c] = 1.f / sd;
            }
            const float sc = buf[off + 2 * MLP_IN];
            if (!(sc > 0.f)) return fail(h, LIMA_ERR_INVALID_ARG, "output scale must be > 0");
            m.out_scale = sc;
            CK(cudaMemcpy(h->lp_mean, m.in_mean, MLP_IN * 4, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(h->lp_invstd, inv.data(), MLP_IN * 4, cudaMemcpyHostToDevice));
            mlp_sync_bf16(m, h->s_main);
            CK(cudaStreamSynchronize(h->s_main));
            h->lp_norm = true;
        }
        return LIMA_OK;
    });
}

int lima_learned_pme_gradients(lima_engine* h, int rows, const float* x, const float* t, float* grads,
                               double* loss) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (rows < 1 || !x || !t || !grads) return fail(h, LIMA_ERR_INVALID_ARG, "bad gradient-check arguments");
    return guarded(h, [&]() {
        if (int e = learned_ready(h)) return e;
        if (rows > h->batch_cap) return fail(h, LIMA_ERR_INVALID_ARG, "more than 65536 rows");
        cudaStream_t s = h->s_main;
        CK(cudaMemcpyAsync(h->batch_raw, x, (size_t)rows * MLP_IN * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(h->batch_T, t, (size_t)rows * 3 * 4, cudaMemcpyHostToDevice, s));
        h->launches += launch_rows_to_bf16(rows, h->batch_raw, h->batch_X, s);
        CK(cudaMemsetAsync(h->d_loss, 0, sizeof(double), s));
        h->launches += mlp_train_step(h->mlp, rows, h->batch_X, h->batch_T, h->acts, 0.f, h->d_loss, s);
        size_t off = 0;
        for (int l = 0; l < 4; ++l) {
            const size_t nw = (size_t)MLP_K[l] * MLP_N[l], nb = MLP_N[l];
            CK(cudaMemcpyAsync(grads + off, h->mlp.gw[l], nw * 4, cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(grads + off + nw, h->mlp.gb[l], nb * 4, cudaMemcpyDeviceToHost, s));
            off += nw + nb;
        }
        double sum = 0.0;
        CK(cudaMemcpyAsync(&sum, h->d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (loss) *loss = sum / (3.0 * rows);
        return LIMA_OK;
    });
}

// ------------------------------------------------------------ thermostat, log
int lima_autotune(lima_engine* h, int periods, int* shape) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (periods < 1) return fail(h, LIMA_ERR_INVALID_ARG, "periods must be >= 1");
    return guarded(h, [&]() {
        ensure_built(h);
        const int pick = h->autotune(periods);
        if (shape) *shape = pick;
        return LIMA_OK;
    });
}

int lima_set_pair_shape(lima_engine* h, int shape) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (shape < 0 || shape > 11 || ((shape & 8) && (shape & 4)))
        return fail(h, LIMA_ERR_INVALID_ARG, "pair kernel shape must be 0-11 (bit 2 only without bit 3)");
    h->nb_shape = shape;
    h->drop_graph();
    return LIMA_OK;
}

int lima_get_thermostat(lima_engine* h, double* temperature, double* scale, int64_t* step) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    const bool have = h->built && h->cur < (int)h->therm_T.size();
    if (temperature) *temperature = have ? h->therm_T[h->cur] : 0.0;
    if (scale) *scale = have ? h->therm_scale[h->cur] : h->p.thermostat_scalar;
    if (step) *step = have ? h->therm_step : -1;
    return LIMA_OK;
}

int lima_get_log(lima_engine* h, int64_t first, int64_t max_frames, int64_t* steps, float* pos_epot,
                 float* force_speed, int64_t* n_frames) {
    if (!h || first < 0 || max_frames < 0) return LIMA_ERR_INVALID_ARG;
    return guarded(h, [&]() {
        if (h->built) h->flush_log();
        const int64_t total = (int64_t)h->log_host_steps.size();
        if (n_frames) *n_frames = total;
        const size_t N = h->built ? (size_t)h->st.n_atoms : 0;
        const int off = h->n_atoms_off.empty() ? 0 : h->n_atoms_off[h->cur];
        const int n = h->sys[h->cur].n;
        for (int64_t f = 0; f < max_frames && first + f < total; ++f) {
            const size_t fr = (size_t)(first + f);
            if (steps) steps[f] = h->log_host_steps[fr];
            for (int a = 0; a < n; ++a) {
                const float4 pe = h->log_host_pe[fr * N + off + a];
                const float4 fs = h->log_host_fs[fr * N + off + a];
                const size_t o = ((size_t)f * n + a) * 4;
                if (pos_epot) pos_epot[o] = pe.x, pos_epot[o + 1] = pe.y, pos_epot[o + 2] = pe.z, pos_epot[o + 3] = pe.w;
                if (force_speed)
                    force_speed[o] = fs.x, force_speed[o + 1] = fs.y, force_speed[o + 2] = fs.z, force_speed[o + 3] = fs.w;
            }
        }
        return LIMA_OK;
    });
}

int lima_clear_log(lima_engine* h) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    h->log_host_pe.clear();
    h->log_host_fs.clear();
    h->log_host_steps.clear();
    h->log_host_pe.shrink_to_fit();
    h->log_host_fs.shrink_to_fit();
    return LIMA_OK;
}

int lima_learned_pme_predict(lima_engine* h, int rows, const float* features, float* out, int impl) {
    if (!h) return LIMA_ERR_INVALID_ARG;
    if (rows < 1 || !features || !out || impl < 0 || impl > 2)
        return fail(h, LIMA_ERR_INVALID_ARG, "bad prediction arguments");
    return guarded(h, [&]() {
        if (int e = learned_ready(h)) return e;
        if (rows > h->batch_cap) return fail(h, LIMA_ERR_INVALID_ARG, "more than 65536 rows");
        cudaStream_t s = h->s_main;
        CK(cudaMemcpyAsync(h->batch_raw, features, (size_t)rows * MLP_IN * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(h->mlp.tc_err, 0, sizeof(int), s));
        if (impl == 0 || impl == 2)
            h->launches += mlp_infer_tc(h->mlp, rows, h->batch_raw, h->lp_mean, h->lp_invstd, h->acts.y, h->mlp.tc_err, s,
                                        impl == 2 ? 1 : 0);
        else
            h->launches += mlp_infer(h->mlp, rows, h->batch_raw, h->lp_mean, h->lp_invstd, h->acts.y, s);
        std::vector<float> y((size_t)rows * 8);
        int err = 0;
        CK(cudaMemcpyAsync(y.data(), h->acts.y, y.size() * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&err, h->mlp.tc_err, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        CK(cudaGetLastError());
        if (err) return fail(h, LIMA_ERR_TIMEOUT, "tensor-core inference: a bounded wait gave up");
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < 3; ++c) out[(size_t)r * 3 + c] = y[(size_t)r * 8 + c];
        return LIMA_OK;
    });
}

}  // extern "C"
