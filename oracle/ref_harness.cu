// ref_harness.cu — TEST INFRASTRUCTURE ONLY.  Evaluates the reference's own
// per-term device functions on inputs read from a file, so that the CPU
// oracle can be checked against the reference's compiled arithmetic.
//
// The reference's headers are compiled from where they lie in the reference
// tree (include paths given by oracle/Makefile's `ref` target, which builds
// this file into oracle/_ref/ref_terms with the reference's own flags:
// -use_fast_math -O3, code/LIMA_ENGINE/CMakeLists.txt:29).  Nothing here is
// part of the library; the binary is run only to generate the golden vectors
// under tests/golden/ (tests/golden/make_ref_golden.py).
//
// Functions evaluated (one GPU thread per sample):
//   lj        LJ::calcLJForceOptim<true,false>     LennardJonesInteractions.cuh:74-108
//   lj_em     LJ::calcLJForceOptim<false,true>     (EM clamp + ForceActivationFunction(.,100))
//   coulomb   PhysicsUtilsDevice::CalcCoulumbForce_optim / CalcCoulumbPotential_optim
//                                                   DeviceAlgorithmsPrivate.cuh:38-95
//   bond      calcSinglebondForces<false>          ForceComputations.cuh:17-51
//   bond_em   calcSinglebondForces<true>
//   angle     calcAnglebondForces (Urey-Bradley)   ForceComputations.cuh:53-115
//   dihedral  calcDihedralbondForces               ForceComputations.cuh:119-210
//   improper  calcImproperdihedralbondForces       ForceComputations.cuh:214-264
//   bspline   LAL::CalcBspline                     DeviceAlgorithmsPrivate.cuh:7-30
//   vvs       EngineUtils::integratePositionVVS / integrateVelocityVVS
//                                                   EngineUtils.cuh:31-41
//   activate  EngineUtils::ForceActivationFunction EngineUtils.cuh:112-140
//   adam      EngineUtils::IntegratePositionADAM   EngineUtils.cuh:44-72
//   interact  canCompoundsInteract<PeriodicBoundaryCondition>
//                                                   Neighborlists.cuh:64-79
//   green     PrecomputeGreensFunctionKernel       PME.cuh:434-495
//
// Usage: ref_terms <kind> <n> <in.f32> <out.f32> [p0 [p1 [p2]]]
// Inputs are float32 records; outputs float32 records (integer results are
// stored as their int32 bit patterns).  Every input is checked on the host
// before the launch: non-finite values and force magnitudes that could reach
// the reference's trap on NaN forces (EngineUtils.cuh:119-122) are refused.
#include "Engine.cuh"
#include "EngineBodies.cuh"
#include "Neighborlists.cuh"
#include "BoundaryCondition.cuh"
#include "SimulationDevice.cuh"
#include "LimaPositionSystem.cuh"
#include "EngineKernels.cuh"
#include "PME.cuh"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

// One out-of-line reference function is referenced by inline code these
// headers emit (file lookup of the install directory); nothing evaluated here
// calls it.
namespace FileUtils {
fs::path GetLimaDir() { return fs::path("."); }
}  // namespace FileUtils

namespace refh {

__device__ inline Float3 ld3(const float* p) { return Float3{p[0], p[1], p[2]}; }
__device__ inline void st3(float* p, const Float3& v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}

__global__ void k_lj(int n, const float* in, float* out) {  // in: dx dy dz sigma eps
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 5 * t;
    const Float3 diff = ld3(a);
    float pot = 0.f;
    const Float3 f = LJ::calcLJForceOptim<true, false>(diff, 1.f / diff.lenSquared(), pot, a[3], a[4],
                                                       LJ::CalcLJOrigin::ComComInter) * 24.f;
    st3(out + 4 * t, f);
    out[4 * t + 3] = pot;
}

__global__ void k_lj_em(int n, const float* in, float* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 5 * t;
    const Float3 diff = ld3(a);
    float pot = 0.f;
    const Float3 f = LJ::calcLJForceOptim<false, true>(diff, 1.f / diff.lenSquared(), pot, a[3], a[4],
                                                       LJ::CalcLJOrigin::ComComInter) * 24.f;
    st3(out + 3 * t, f);
}

__global__ void k_coulomb(int n, const float* in, float* out) {  // in: q1 q2 dx dy dz
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 5 * t;
    const Float3 diff = ld3(a + 2);
    const Float3 f = PhysicsUtilsDevice::CalcCoulumbForce_optim(a[0] * a[1], diff);
    const float pot = PhysicsUtilsDevice::CalcCoulumbPotential_optim(a[0], a[1], diff);
    st3(out + 4 * t, f);
    out[4 * t + 3] = pot;
}

template <bool EM>
__global__ void k_bond(int n, const float* in, float* out) {  // in: pa(3) pb(3) b0 kb
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 8 * t;
    SingleBond::Parameters p;
    p.b0 = a[6];
    p.kb = a[7];
    Float3 r[2];
    float pot = 0.f;
    LimaForcecalc::calcSinglebondForces<EM>(ld3(a), ld3(a + 3), p, r, pot, false);
    st3(out + 7 * t, r[0]);
    st3(out + 7 * t + 3, r[1]);
    out[7 * t + 6] = pot;
}

// the bond structs' constructors are host-only: they are filled on the host
// from the inputs' parameters and copied to the device (make_terms below)
__global__ void k_angle(int n, const float* in, const AngleUreyBradleyBond* bt, float* out) {
    // in: p0 p1 p2 (9) theta0 kTheta ub0 kUB
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 13 * t;
    Float3 r[3];
    float pot = 0.f;
    LimaForcecalc::calcAnglebondForces(ld3(a), ld3(a + 3), ld3(a + 6), bt[t], r, pot);
    for (int k = 0; k < 3; ++k) st3(out + 10 * t + 3 * k, r[k]);
    out[10 * t + 9] = pot;
}

__global__ void k_dihedral(int n, const float* in, const DihedralBond* bt, float* out) {
    // in: p0..p3 (12) phi0 kphi n
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 15 * t;
    Float3 r[4];
    float pot = 0.f;
    LimaForcecalc::calcDihedralbondForces(ld3(a), ld3(a + 3), ld3(a + 6), ld3(a + 9), bt[t], r, pot);
    for (int k = 0; k < 4; ++k) st3(out + 13 * t + 3 * k, r[k]);
    out[13 * t + 12] = pot;
}

__global__ void k_improper(int n, const float* in, const ImproperDihedralBond* bt, float* out) {
    // in: p0..p3 (12) psi0 kpsi
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 14 * t;
    Float3 r[4];
    float pot = 0.f;
    LimaForcecalc::calcImproperdihedralbondForces(ld3(a), ld3(a + 3), ld3(a + 6), ld3(a + 9), bt[t], r, pot);
    for (int k = 0; k < 4; ++k) st3(out + 13 * t + 3 * k, r[k]);
    out[13 * t + 12] = pot;
}

__global__ void k_bspline(int n, const float* in, float* out) {  // in: f
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    LAL::CalcBspline(in[t], out + 4 * t);
}

// in: vel_prev(3) force_prev(3) force(3) mass dt  ->  position step (Coord, 3 x int32), velocity (3)
__global__ void k_vvs(int n, const float* in, float* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 11 * t;
    const Float3 vprev = ld3(a), fprev = ld3(a + 3), f = ld3(a + 6);
    // the order of CompoundIntegrationKernel (EngineKernels.cuh:400-403): the
    // position step takes the updated velocity
    const Float3 v = EngineUtils::integrateVelocityVVS(vprev, fprev, f, a[10], a[9]);
    const Coord step = EngineUtils::integratePositionVVS(Coord{0, 0, 0}, v, f, a[9], a[10]);
    out[6 * t + 0] = __int_as_float(step.x);
    out[6 * t + 1] = __int_as_float(step.y);
    out[6 * t + 2] = __int_as_float(step.z);
    st3(out + 6 * t + 3, v);
}

__global__ void k_activate(int n, const float* in, float* out) {  // in: force(3) scalar
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 4 * t;
    st3(out + 3 * t, EngineUtils::ForceActivationFunction(ld3(a), a[3]));
}

// in: force(3) m(3) v(3) step  ->  position step (Coord, 3 x int32), m'(3), v'(3)
__global__ void k_adam(int n, const float* in, float* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 10 * t;
    AdamState s{ld3(a + 3), ld3(a + 6)};
    const Coord c = EngineUtils::IntegratePositionADAM(Coord{0, 0, 0}, ld3(a), &s, (int)a[9]);
    out[9 * t + 0] = __int_as_float(c.x);
    out[9 * t + 1] = __int_as_float(c.y);
    out[9 * t + 2] = __int_as_float(c.z);
    st3(out + 9 * t + 3, s.firstMoment);
    st3(out + 9 * t + 6, s.secondMoment);
}

// in: left key positions (6), right key positions (6), left radii (2), right radii (2)
__global__ void k_interact(int n, const float* in, float* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* a = in + 16 * t;
    CompoundInteractionBoundary l{}, r{};
    l.radii[0] = a[12];
    l.radii[1] = a[13];
    r.radii[0] = a[14];
    r.radii[1] = a[15];
    const Float3 pl[2] = {ld3(a), ld3(a + 3)}, pr[2] = {ld3(a + 6), ld3(a + 9)};
    out[t] = canCompoundsInteract<PeriodicBoundaryCondition>(l, r, pl, pr) ? 1.f : 0.f;
}

// per-sample bond structs from the parameters at offset `off` of each input record
template <class T, class F>
T* make_terms(const std::vector<float>& in, int n, int rec, F&& fill) {
    std::vector<T> h(n);
    for (int t = 0; t < n; ++t) fill(h[t], &in[(size_t)rec * t]);
    T* d = nullptr;
    if (cudaMalloc(&d, sizeof(T) * (size_t)n) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, h.data(), sizeof(T) * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    return d;
}

bool finite_all(const std::vector<float>& v) {
    for (float x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

int fail(const char* msg) {
    std::fprintf(stderr, "ref_terms: %s\n", msg);
    return 2;
}

#define CK(x)                                                                              \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            std::fprintf(stderr, "ref_terms: %s: %s\n", #x, cudaGetErrorString(e_));      \
            return 3;                                                                      \
        }                                                                                  \
    } while (0)

}  // namespace refh
using namespace refh;

int main(int argc, char** argv) {
    if (argc < 5) return fail("usage: ref_terms <kind> <n> <in.f32> <out.f32> [p0 [p1 [p2]]]");
    const std::string kind = argv[1];
    const int n = std::atoi(argv[2]);
    const double p0 = argc > 5 ? std::atof(argv[5]) : 0.0;
    const double p1 = argc > 6 ? std::atof(argv[6]) : 0.0;
    struct K {
        const char* name;
        int in, out;
    };
    const K kinds[] = {{"lj", 5, 4},       {"lj_em", 5, 3},    {"coulomb", 5, 4}, {"bond", 8, 7},
                       {"bond_em", 8, 7},  {"angle", 13, 10},  {"dihedral", 15, 13}, {"improper", 14, 13},
                       {"bspline", 1, 4},  {"vvs", 11, 6},     {"activate", 4, 3}, {"adam", 10, 9},
                       {"interact", 16, 1}, {"green", 0, 0}};
    const K* k = nullptr;
    for (const K& c : kinds)
        if (kind == c.name) k = &c;
    if (!k) return fail("unknown kind");

    if (kind == "green") {
        // n = grid points per dimension, p0 = box length [nm], p1 = Ewald kappa [1/nm]
        if (n < 4 || n > 256 || !(p0 > 0.0) || !(p1 > 0.0)) return fail("bad green arguments");
        const int total = (n / 2 + 1) * n * n;
        float* d = nullptr;
        CK(cudaMalloc(&d, (size_t)total * sizeof(float)));
        PrecomputeGreensFunctionKernel<<<(total + 255) / 256, 256>>>(d, n, p0, p1);
        CK(cudaGetLastError());
        std::vector<float> h(total);
        CK(cudaMemcpy(h.data(), d, (size_t)total * sizeof(float), cudaMemcpyDeviceToHost));
        CK(cudaFree(d));
        FILE* fo = std::fopen(argv[4], "wb");
        if (!fo || std::fwrite(h.data(), sizeof(float), h.size(), fo) != h.size()) return fail("write failed");
        std::fclose(fo);
        return 0;
    }

    if (n <= 0 || n > (1 << 22)) return fail("bad sample count");
    std::vector<float> in((size_t)n * k->in);
    FILE* fi = std::fopen(argv[3], "rb");
    if (!fi || std::fread(in.data(), sizeof(float), in.size(), fi) != in.size()) return fail("read failed");
    std::fclose(fi);
    if (!finite_all(in)) return fail("non-finite input");
    // the reference traps on a NaN force and draws a random force for an
    // infinite one (EngineUtils.cuh:112-123): keep every force far from both
    if (kind == "activate") {
        for (int t = 0; t < n; ++t) {
            const float* a = &in[(size_t)4 * t];
            const double f2 = (double)a[0] * a[0] + (double)a[1] * a[1] + (double)a[2] * a[2];
            if (!(f2 < 1e30) || !(a[3] > 0.f)) return fail("activate input out of range");
        }
    }
    if (kind == "lj_em" || kind == "lj") {
        for (int t = 0; t < n; ++t) {
            const float* a = &in[(size_t)5 * t];
            const double r2 = (double)a[0] * a[0] + (double)a[1] * a[1] + (double)a[2] * a[2];
            if (!(r2 >= 0.01 && r2 < 16.0) || !(a[3] > 0.f && a[3] < 0.6f) || !(a[4] >= 0.f && a[4] < 1e4f))
                return fail("lj input out of range");
        }
    }
    if (kind == "coulomb") {
        for (int t = 0; t < n; ++t) {
            const float* a = &in[(size_t)5 * t];
            const double r2 = (double)a[2] * a[2] + (double)a[3] * a[3] + (double)a[4] * a[4];
            if (!(r2 >= 0.01)) return fail("coulomb input out of range");
        }
    }

    if (kind == "coulomb" || kind == "interact") {
        // Ewald kappa (0 = plain Coulomb: erfc(0) = 1), cutoff, integer box size
        const float kappa = (float)p0, cutoff = (float)(p1 > 0.0 ? p1 : 1.0);
        CK(cudaMemcpyToSymbol(DeviceConstants::ewaldKappa, &kappa, sizeof(float)));
        CK(cudaMemcpyToSymbol(DeviceConstants::cutoffNM, &cutoff, sizeof(float)));
        BoxSize bs;
        bs.Set(argc > 7 ? std::atoi(argv[7]) : 10);
        CK(cudaMemcpyToSymbol(DeviceConstants::boxSize, &bs, sizeof(BoxSize)));
    }

    float *din = nullptr, *dout = nullptr;
    CK(cudaMalloc(&din, in.size() * sizeof(float)));
    CK(cudaMalloc(&dout, (size_t)n * k->out * sizeof(float)));
    CK(cudaMemcpy(din, in.data(), in.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemset(dout, 0, (size_t)n * k->out * sizeof(float)));
    const int tb = 128, nb = (n + tb - 1) / tb;
    if (kind == "lj") k_lj<<<nb, tb>>>(n, din, dout);
    else if (kind == "lj_em") k_lj_em<<<nb, tb>>>(n, din, dout);
    else if (kind == "coulomb") k_coulomb<<<nb, tb>>>(n, din, dout);
    else if (kind == "bond") k_bond<false><<<nb, tb>>>(n, din, dout);
    else if (kind == "bond_em") k_bond<true><<<nb, tb>>>(n, din, dout);
    else if (kind == "angle") {
        AngleUreyBradleyBond* bt = make_terms<AngleUreyBradleyBond>(in, n, 13, [](AngleUreyBradleyBond& b, const float* a) {
            b.params.theta0 = a[9];
            b.params.kTheta = a[10];
            b.params.ub0 = a[11];
            b.params.kUB = a[12];
        });
        if (!bt) return fail("bond structs");
        k_angle<<<nb, tb>>>(n, din, bt, dout);
    } else if (kind == "dihedral") {
        DihedralBond* bt = make_terms<DihedralBond>(in, n, 15, [](DihedralBond& b, const float* a) {
            b.params.phi_0 = a[12];
            b.params.k_phi = a[13];
            b.params.n = a[14];
        });
        if (!bt) return fail("bond structs");
        k_dihedral<<<nb, tb>>>(n, din, bt, dout);
    } else if (kind == "improper") {
        ImproperDihedralBond* bt = make_terms<ImproperDihedralBond>(in, n, 14, [](ImproperDihedralBond& b, const float* a) {
            b.params.psi_0 = a[12];
            b.params.k_psi = a[13];
        });
        if (!bt) return fail("bond structs");
        k_improper<<<nb, tb>>>(n, din, bt, dout);
    }
    else if (kind == "bspline") k_bspline<<<nb, tb>>>(n, din, dout);
    else if (kind == "vvs") k_vvs<<<nb, tb>>>(n, din, dout);
    else if (kind == "activate") k_activate<<<nb, tb>>>(n, din, dout);
    else if (kind == "adam") k_adam<<<nb, tb>>>(n, din, dout);
    else if (kind == "interact") k_interact<<<nb, tb>>>(n, din, dout);
    CK(cudaGetLastError());
    std::vector<float> out((size_t)n * k->out);
    CK(cudaMemcpy(out.data(), dout, out.size() * sizeof(float), cudaMemcpyDeviceToHost));
    CK(cudaFree(din));
    CK(cudaFree(dout));
    FILE* fo = std::fopen(argv[4], "wb");
    if (!fo || std::fwrite(out.data(), sizeof(float), out.size(), fo) != out.size()) return fail("write failed");
    std::fclose(fo);
    return 0;
}
