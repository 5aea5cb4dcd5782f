// lima_oracle.cpp — CPU restatement of LIMA's force/integration formulas.
// TEST INFRASTRUCTURE ONLY (see lima_oracle.h): used by tests/, the smoke check
// and the CPU-baseline leg of bench.py; never linked into the product library.
//
// Every function states the reference file:line whose arithmetic it restates.
// The code is written from those formulas, not copied.
#include "lima_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Constants.h:43-60 and PhysicsUtils.cuh:5 — k_e = COULOMBCONSTANT/NANO/N_A*KILO*KILO
constexpr double kCoulomb = 8.9875517873681764e9 / 1e-9 / 6.02214076e23 * 1000.0 * 1000.0;
constexpr double kEtoKCmol = 1.602176634e-19 * 6.02214076e23 / 1000.0;
constexpr double kPi = 3.14159265358979323846;
constexpr double kPiRef = 3.14159;  // Constants.h:51 (truncated)

template <typename T>
struct V3 {
    T x, y, z;
};
template <typename T>
inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T>
inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T>
inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T>
inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename T>
inline T len(V3<T> a) { return std::sqrt(dot(a, a)); }
template <typename T>
inline V3<T> unit(V3<T> a) {
    T l = len(a);
    return l != T(0) ? a * (T(1) / l) : V3<T>{0, 0, 0};
}

using D3 = V3<double>;

inline D3 load(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline void addf(double* f, int i, D3 v) {
    f[3 * i] += v.x;
    f[3 * i + 1] += v.y;
    f[3 * i + 2] += v.z;
}

template <typename T>
inline T min_image_1(T d, T L) {
    if (L <= T(0)) return d;
    return d - L * std::nearbyint(d / L);
}
template <typename T>
inline V3<T> min_image(V3<T> d, const T* L) {
    if (!L) return d;
    return {min_image_1(d.x, L[0]), min_image_1(d.y, L[1]), min_image_1(d.z, L[2])};
}

inline bool is_excluded(const int* off, const int* idx, int i, int j) {
    if (!off) return false;
    for (int k = off[i]; k < off[i + 1]; ++k)
        if (idx[k] == j) return true;
    return false;
}

// ------------------------------------------------------------------ cell grid
// A plain linked-cell grid with cells no smaller than rc; used only to make the
// all-pairs search affordable at 1e5 atoms.  Falls back to all pairs when a
// dimension has fewer than 3 cells.
struct CellGrid {
    int nc[3] = {0, 0, 0};
    bool ok = false;
    std::vector<int> head, next;
    void build(int n, const double* pos, const double* box, double rc) {
        ok = false;
        if (!box) return;
        for (int d = 0; d < 3; ++d) {
            nc[d] = (int)std::floor(box[d] / rc);
            if (nc[d] < 3) return;
        }
        ok = true;
        head.assign((size_t)nc[0] * nc[1] * nc[2], -1);
        next.assign(n, -1);
        for (int i = 0; i < n; ++i) {
            int c = cell_of(pos + 3 * i, box);
            next[i] = head[c];
            head[c] = i;
        }
    }
    int coord(double x, double L, int n) const {
        double u = x / L;
        u -= std::floor(u);
        int c = (int)(u * n);
        return c >= n ? n - 1 : (c < 0 ? 0 : c);
    }
    int cell_of(const double* p, const double* box) const {
        int cx = coord(p[0], box[0], nc[0]), cy = coord(p[1], box[1], nc[1]),
            cz = coord(p[2], box[2], nc[2]);
        return cx + nc[0] * (cy + nc[1] * cz);
    }
    // calls fn(j) for every atom in the 27 cells around atom position p
    template <typename F>
    void visit(const double* p, const double* box, F&& fn) const {
        int c0[3] = {coord(p[0], box[0], nc[0]), coord(p[1], box[1], nc[1]),
                     coord(p[2], box[2], nc[2])};
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int cx = (c0[0] + dx + nc[0]) % nc[0];
                    int cy = (c0[1] + dy + nc[1]) % nc[1];
                    int cz = (c0[2] + dz + nc[2]) % nc[2];
                    for (int j = head[cx + nc[0] * (cy + nc[1] * cz)]; j >= 0; j = next[j]) fn(j);
                }
    }
};

// ----------------------------------------------------------- pair interaction
// LJ: LennardJonesInteractions.cuh:74-108 (force on i, diff = r_j - r_i).
// Coulomb: DeviceAlgorithmsPrivate.cuh:38-95 with the 2 kappa/sqrt(pi) r exp(-k^2r^2) term.
template <typename T>
struct PairOut {
    V3<T> f_on_i;
    T e_lj, e_coul;
};

template <typename T>
inline PairOut<T> pair_interaction(V3<T> diff /* r_j - r_i */, T r2, T sig, T eps, T qq, int es_mode,
                                   T kappa, T ke, T pi_c, bool em = false) {
    PairOut<T> o;
    const T inv_r2 = T(1) / r2;
    T s = sig * sig * inv_r2;
    s = s * s * s;
    T lj_scalar = T(24) * eps * s * inv_r2 * (T(1) - T(2) * s);  // attractive when positive
    if (em) {
        // energy-minimisation variant (LennardJonesInteractions.cuh:85-101): the
        // scalar is bounded by +-1e20 in the reference's 1/24 J/mol/nm unit, then
        // the pair force passes through ForceActivationFunction(force, 100)
        // (EngineUtils.cuh:112-140): |F| -> A tanh(|F|/A), A = 1e3 * 1e3 * 100 in
        // that unit; the 1e-8 guard of its division is in the same unit
        const T A = T(24) * T(1e8);
        lj_scalar = std::fmax(std::fmin(lj_scalar, T(24) * T(1e20)), -T(24) * T(1e20));
        const T f = std::fabs(lj_scalar) * std::sqrt(r2);
        lj_scalar *= A * std::tanh(f / A) / (f + T(24) * T(1e-8));
    }
    o.e_lj = T(4) * eps * s * (s - T(1));
    T coul_scalar = T(0);  // multiplies (r_i - r_j)
    o.e_coul = T(0);
    if (es_mode != 0 && qq != T(0)) {
        const T r = std::sqrt(r2);
        const T inv_r = T(1) / r;
        T fs = qq * inv_r * inv_r * inv_r;
        T es = qq * inv_r;
        if (es_mode == 2) {
            const T kr = kappa * r;
            const T erfc_kr = std::erfc(kr);
            fs *= erfc_kr + T(2) * kappa / std::sqrt(pi_c) * r * std::exp(-kr * kr);
            es *= erfc_kr;
        }
        coul_scalar = fs * ke;
        o.e_coul = es * ke;
    }
    // F_i = lj_scalar * (r_j - r_i) + coul_scalar * (r_i - r_j)
    o.f_on_i = diff * (lj_scalar - coul_scalar);
    return o;
}

template <typename T>
int64_t nonbonded_impl(int n, const double* pos, const double* box, const double* q,
                       const double* sigma, const double* eps, const int* eo, const int* ei,
                       double rc, int es_mode, double kappa, int nthreads, double* forces,
                       double* energies, double* atom_energy = nullptr, bool em = false) {
    CellGrid grid;
    grid.build(n, pos, box, rc);
    const T rcT = (T)rc;
    const T rc2 = rcT * rcT;
    const T inv_rc2 = T(1) / rc2;
    const T ke = (T)kCoulomb;
    const T pi_c = sizeof(T) == 4 ? (T)kPiRef : (T)kPi;
    T boxT[3] = {box ? (T)box[0] : T(0), box ? (T)box[1] : T(0), box ? (T)box[2] : T(0)};
    const T* Lp = box ? boxT : nullptr;
    double e_lj = 0, e_coul = 0, vir = 0;
    int64_t npairs = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : e_lj, e_coul, vir, npairs)
#endif
    for (int i = 0; i < n; ++i) {
        const V3<T> pi{(T)pos[3 * i], (T)pos[3 * i + 1], (T)pos[3 * i + 2]};
        const T qi = (T)q[i], si = (T)sigma[i], epi = (T)eps[i];
        V3<T> fi{0, 0, 0};
        double el = 0, ec = 0, vr = 0;
        int64_t np = 0;
        auto body = [&](int j) {
            if (j == i) return;
            if (is_excluded(eo, ei, i, j)) return;
            const V3<T> pj{(T)pos[3 * j], (T)pos[3 * j + 1], (T)pos[3 * j + 2]};
            const V3<T> diff = min_image(pj - pi, Lp);
            const T r2 = dot(diff, diff);
            // the reference's cutoff test compares reciprocals (EngineUtils.cuh:175-180)
            if (sizeof(T) == 4) {
                if (T(1) / r2 < inv_rc2) return;
            } else if (r2 > rc2) {
                return;
            }
            const T sig = (si + (T)sigma[j]) * T(0.5);
            const T ep = std::sqrt(epi * (T)eps[j]);
            PairOut<T> o = pair_interaction<T>(diff, r2, sig, ep, qi * (T)q[j], es_mode, (T)kappa, ke, pi_c, em);
            fi = fi + o.f_on_i;
            el += 0.5 * (double)o.e_lj;
            ec += 0.5 * (double)o.e_coul;
            vr += 0.5 * 0.5 * (double)dot(diff, o.f_on_i);  // -1/2 r_ij.f_ij with r_ij = -diff
            if (j > i) ++np;
        };
        if (grid.ok) {
            grid.visit(pos + 3 * i, box, body);
        } else {
            for (int j = 0; j < n; ++j) body(j);
        }
        forces[3 * i] += (double)fi.x;
        forces[3 * i + 1] += (double)fi.y;
        forces[3 * i + 2] += (double)fi.z;
        if (atom_energy) atom_energy[i] += el + ec;  // half of every pair energy of atom i
        e_lj += el;
        e_coul += ec;
        vir += vr;
        npairs += np;
    }
    if (energies) {
        energies[0] += e_lj;
        energies[1] += e_coul;
        energies[2] += vir;
    }
    return npairs;
}

// ------------------------------------------------------------------ bonded
// ForceComputations.cuh:17-51 — harmonic bond, force on a = -kb (|d|-b0) d/|d|, d = a-b
void bond_term(D3 a, D3 b, double b0, double kb, D3* f, double* e) {
    const D3 d = a - b;
    const double r = len(d);
    const double err = r - b0;
    *e = 0.5 * kb * err * err;
    const D3 u = unit(d);
    f[0] = u * (-kb * err);
    f[1] = u * (kb * err);
}

// ForceComputations.cuh:53-115 — harmonic angle with forces along the in-plane
// normals of each arm, plus the Urey-Bradley 1-3 spring.
void angle_term(D3 l, D3 m, D3 r, const double* p, D3* f, double* e) {
    const double theta0 = p[0], kt = p[1], ub0 = p[2], kub = p[3];
    const D3 a1 = l - m, a2 = r - m;
    const D3 v1 = unit(a1), v2 = unit(a2);
    const D3 nrm = unit(cross(v1, v2));
    const D3 dir_l = unit(cross(nrm, v1));  // = v1 x (-n): in-plane, towards the other arm
    const D3 dir_r = unit(cross(v2, nrm));
    double c = dot(v1, v2);
    c = std::min(1.0, std::max(-1.0, c));
    const double theta = std::acos(c);
    const double err = theta - theta0;
    const double torque = kt * err;
    f[0] = dir_l * (torque / len(a1));
    f[2] = dir_r * (torque / len(a2));
    f[1] = (f[0] + f[2]) * -1.0;
    double en = 0.5 * kt * err * err;
    // Urey-Bradley spring between the outer atoms
    const D3 d13 = l - r;
    const double e13 = len(d13) - ub0;
    en += 0.5 * kub * e13 * e13;
    const D3 u13 = unit(d13);
    f[0] = f[0] + u13 * (-kub * e13);
    f[2] = f[2] + u13 * (kub * e13);
    *e = en;
}

// ForceComputations.cuh:119-210 — periodic dihedral k(1+cos(n*tau - phi0)) with
// tau = -atan2(sin, cos); gradients through cos(phi) when |sin phi| > 0.1, else
// through sin(phi) (the switch that keeps both branches well conditioned).
void dihedral_term(D3 p0, D3 p1, D3 p2, D3 p3, const double* p, D3* f, double* e) {
    const double phi0 = p[0], kphi = p[1], mult = p[2];
    const D3 b1 = p1 - p0, b2 = p2 - p1, b3 = p3 - p2;
    D3 A = cross(b1, b2), B = cross(b2, b3), C = cross(b2, A);
    const double iA = 1.0 / len(A), iB = 1.0 / len(B), iC = 1.0 / len(C);
    const double cphi = dot(A, B) * iA * iB;
    const double sphi = dot(C, B) * iC * iB;
    const double tau = -std::atan2(sphi, cphi);
    *e = kphi * (1.0 + std::cos(mult * tau - phi0));
    const double torque = kphi * mult * std::sin(mult * tau - phi0);
    const D3 Bn = B * iB;
    D3 g1, g2, g3;
    if (std::fabs(sphi) > 0.1) {
        const D3 An = A * iA;
        const D3 dA = (An * cphi - Bn) * iA;  // d cos / d A
        const D3 dB = (Bn * cphi - An) * iB;  // d cos / d B
        const double s = torque / sphi;
        g1 = cross(b2, dA) * s;
        g3 = cross(b2, dB) * (-s);
        g2 = (cross(b3, dB) - cross(b1, dA)) * s;
    } else {
        const D3 Cn = C * iC;
        const D3 dC = (Cn * sphi - Bn) * iC;  // d sin / d C
        const D3 dB = (Bn * sphi - Cn) * iB;  // d sin / d B
        const double s = -torque / cphi;
        // C = b2 x (b1 x b2): its gradient wrt b1 is the projection b2 x (dC x b2)
        g1 = cross(b2, cross(dC, b2)) * s;
        g3 = cross(dB, b2) * s;
        // gradient of C wrt b2 contracted with dC, plus the B = b2 x b3 part
        const D3 t = b2 * (2.0 * dot(b1, dC)) - b1 * dot(b2, dC) - dC * dot(b2, b1);
        g2 = (t + cross(b3, dB)) * s;
    }
    f[0] = g1;
    f[1] = g2 - g1;
    f[2] = g3 - g2;
    f[3] = g3 * -1.0;
}

inline double dist_to_line(D3 pt, D3 a, D3 b) {
    return len(cross(b - a, a - pt)) / len(b - a);
}

// ForceComputations.cuh:214-264 — improper as the signed angle between the
// (i,j,k) and (l,j,k) planes; forces on i and l along the plane normals,
// remainder split over j and k by arm length.
void improper_term(D3 pi, D3 pj, D3 pk, D3 pl, const double* p, D3* f, double* e) {
    const double psi0 = p[0], kpsi = p[1];
    const D3 ij = unit(pj - pi), ik = unit(pk - pi), il = unit(pl - pi);
    const D3 lj = unit(pj - pl), lk = unit(pk - pl);
    const D3 n1 = unit(cross(ij, ik));
    const D3 n2 = unit(cross(lj, lk));
    double c = std::min(1.0, std::max(-1.0, dot(n1, n2)));
    double ang = std::acos(c);
    if (dot(n1, il) > 0.0) ang = -ang;
    const double err = ang - psi0;
    *e = 0.5 * kpsi * err * err;
    const double torque = kpsi * err;
    f[3] = n2 * (torque / dist_to_line(pl, pj, pk));
    f[0] = n1 * (-torque / dist_to_line(pi, pj, pk));
    const D3 rest = (f[0] + f[3]) * -1.0;
    const double lij = len(pj - pi), lik = len(pk - pi);
    const double ratio = lij / (lij + lik);
    f[1] = rest * (1.0 - ratio);
    f[2] = rest * ratio;
}

// ForceComputations.cuh:335-376 — LJ pair bond between two atoms, no cutoff.
void pairbond_term(D3 a, D3 b, double sig, double eps, D3* f, double* e) {
    const D3 diff = b - a;
    const double r2 = dot(diff, diff);
    double s = sig * sig / r2;
    s = s * s * s;
    const double fs = 24.0 * eps * s / r2 * (1.0 - 2.0 * s);
    f[0] = diff * fs;
    f[1] = diff * (-fs);
    *e = 4.0 * eps * s * (s - 1.0);
}

// ------------------------------------------------------------------- FFT
using cd = std::complex<double>;

// recursive mixed-radix DFT (any length).  tw holds exp(sign*2*pi*i*k/N0) for
// the top-level length N0; a sub-transform of length n uses stride N0/n.
void fft1d(cd* x, int n, const cd* tw, int tstride, int N0, std::vector<cd>& scratch) {
    if (n <= 1) return;
    int p = 0;
    for (int f : {2, 3, 5, 7})
        if (n % f == 0) {
            p = f;
            break;
        }
    if (p == 0) {  // prime length: direct DFT
        scratch.assign(x, x + n);
        for (int k = 0; k < n; ++k) {
            cd s = 0;
            for (int j = 0; j < n; ++j) s += scratch[j] * tw[((long long)j * k % n) * tstride];
            x[k] = s;
        }
        return;
    }
    const int m = n / p;
    std::vector<cd> sub((size_t)n);
    for (int r = 0; r < p; ++r)
        for (int j = 0; j < m; ++j) sub[(size_t)r * m + j] = x[j * p + r];
    for (int r = 0; r < p; ++r) fft1d(&sub[(size_t)r * m], m, tw, tstride * p, N0, scratch);
    for (int k = 0; k < n; ++k) {
        cd s = 0;
        for (int r = 0; r < p; ++r) s += sub[(size_t)r * m + (k % m)] * tw[(size_t)((long long)r * k % n) * tstride];
        x[k] = s;
    }
}

std::vector<cd> twiddles(int n, int sign) {
    std::vector<cd> t(n);
    for (int k = 0; k < n; ++k) t[k] = std::polar(1.0, sign * 2.0 * kPi * k / n);
    return t;
}

void fft3d(int nx, int ny, int nz, cd* g, int sign) {
    const std::vector<cd> tx = twiddles(nx, sign), ty = twiddles(ny, sign), tz = twiddles(nz, sign);
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        std::vector<cd> line(std::max(nx, std::max(ny, nz))), scratch;
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y) fft1d(&g[(size_t)nx * (y + (size_t)ny * z)], nx, tx.data(), 1, nx, scratch);
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x) {
                for (int y = 0; y < ny; ++y) line[y] = g[x + (size_t)nx * (y + (size_t)ny * z)];
                fft1d(line.data(), ny, ty.data(), 1, ny, scratch);
                for (int y = 0; y < ny; ++y) g[x + (size_t)nx * (y + (size_t)ny * z)] = line[y];
            }
#ifdef _OPENMP
#pragma omp for collapse(2)
#endif
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                for (int z = 0; z < nz; ++z) line[z] = g[x + (size_t)nx * (y + (size_t)ny * z)];
                fft1d(line.data(), nz, tz.data(), 1, nz, scratch);
                for (int z = 0; z < nz; ++z) g[x + (size_t)nx * (y + (size_t)ny * z)] = line[z];
            }
    }
}

// order-4 cardinal B-spline weights on nodes floor(u)-1..floor(u)+2
// (DeviceAlgorithmsPrivate.cuh:7-30) and their derivatives w.r.t. the fraction
inline void bspline4(double f, double* w, double* dw) {
    const double g = 1.0 - f;
    w[0] = g * g * g / 6.0;
    w[1] = (4.0 - 6.0 * f * f + 3.0 * f * f * f) / 6.0;
    w[2] = (1.0 + 3.0 * f + 3.0 * f * f - 3.0 * f * f * f) / 6.0;
    w[3] = f * f * f / 6.0;
    if (dw) {
        dw[0] = -0.5 * g * g;
        dw[1] = -2.0 * f + 1.5 * f * f;
        dw[2] = 0.5 + f - 1.5 * f * f;
        dw[3] = 0.5 * f * f;
    }
}

inline int wrapi(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// The reference convention's influence function at wave index m
// (PME.cuh:434-495): 4 pi/k^2 e^{-k^2/4 kappa^2} k_e times the squared product
// of sinc^4(k_d h_d / 2), with the truncated pi of Constants.h:51; zero at k = 0.
// Without the N/V factor of the oracle's own normalisation.
inline double influence_ref(const int* m, const double* box, const int* K, double kappa) {
    if (m[0] == 0 && m[1] == 0 && m[2] == 0) return 0.0;
    double kv[3], k2 = 0.0;
    for (int d = 0; d < 3; ++d) {
        kv[d] = 2.0 * kPiRef * m[d] / box[d];
        k2 += kv[d] * kv[d];
    }
    const double g = 4.0 * kPiRef / k2 * std::exp(-k2 / (4.0 * kappa * kappa)) * kCoulomb;
    double s = 1.0;
    for (int d = 0; d < 3; ++d) {
        const double kh = kv[d] * (box[d] / K[d]) * 0.5;
        const double sc = std::fabs(kh) < 1e-14 ? 1.0 : std::sin(kh) / kh;
        s *= sc * sc * sc * sc;
    }
    return g * s * s;
}

// EngineUtils.cuh:112-140 — the energy minimiser's force activation: the force
// is rescaled to length A tanh(|F|/A), A = 1e6 * scalar [J/mol/nm], with the
// reference's 1e-8 guard on the division.
inline void force_activation(const double* f, double scalar, double* out) {
    const double A = 1000.0 * 1000.0 * scalar;
    const double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    const double k = A * std::tanh(fl / A) / (fl + 1e-8);
    for (int d = 0; d < 3; ++d) out[d] = f[d] * k;
}

// EngineUtils.cuh:44-72 — one ADAM move: the force is scaled by 1e-8, the
// moments updated with beta 0.9 / 0.999, bias-corrected at `step`, and the
// position moves by alpha 1e-8 m/(sqrt(v) + 1e-8), alpha = 8000.
inline void adam_move(const double* f, double* m1, double* m2, int step, double* pos) {
    const double alpha = 8000.0, b1 = 0.9, b2 = 0.999, epsn = 1e-8;
    for (int d = 0; d < 3; ++d) {
        const double g = f[d] * 1e-8;
        m1[d] = m1[d] * b1 + g * (1 - b1);
        m2[d] = m2[d] * b2 + g * g * (1 - b2);
        const double mh = m1[d] / (1 - std::pow(b1, step));
        const double vh = m2[d] / (1 - std::pow(b2, step));
        pos[d] += mh / (std::sqrt(vh) + epsn) * alpha * 1e-8;
    }
}

// Neighborlists.cuh:64-79 with LimaPositionSystem.cuh:194-198 and
// BoundaryCondition.cuh:56-65 — two compounds are neighbours when any pair of
// their two key particles is closer than cutoff + radius_left + radius_right.
// The distance is taken in FP32 with the reference's hyper-position rule: the
// right particle moves by one box length along each axis where it lies more
// than half a box away (a strict comparison against L/2), then |left - right|.
inline bool compounds_interact(const double* kl, const double* kr, const double* rl, const double* rr, float L,
                               float cutoff) {
    const float half = L / 2.f;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            float d2 = 0.f;
            for (int c = 0; c < 3; ++c) {
                const float s = (float)kl[3 * a + c];
                float m = (float)kr[3 * b + c];
                m += L * (float)((s - m) > half);
                m -= L * (float)((s - m) < -half);
                const float dd = s - m;
                d2 += dd * dd;
            }
            if (std::sqrt(d2) < cutoff + (float)rl[a] + (float)rr[b]) return true;
        }
    return false;
}

}  // namespace

// ====================================================================== API
extern "C" {

double orc_coulomb_constant(void) { return kCoulomb; }
double orc_e_to_kcmol(void) { return kEtoKCmol; }

int64_t orc_nonbonded(int n, const double* pos, const double* box, const double* q,
                      const double* sigma, const double* eps, const int* excl_off,
                      const int* excl_idx, double rc, int es_mode, double kappa, int precision,
                      int nthreads, double* forces, double* energies) {
    if (precision == 32)
        return nonbonded_impl<float>(n, pos, box, q, sigma, eps, excl_off, excl_idx, rc, es_mode,
                                     kappa, nthreads, forces, energies);
    return nonbonded_impl<double>(n, pos, box, q, sigma, eps, excl_off, excl_idx, rc, es_mode,
                                  kappa, nthreads, forces, energies);
}

int64_t orc_nonbonded_atoms(int n, const double* pos, const double* box, const double* q,
                            const double* sigma, const double* eps, const int* excl_off,
                            const int* excl_idx, double rc, int es_mode, double kappa, int nthreads,
                            double* forces, double* energies, double* atom_energy) {
    return nonbonded_impl<double>(n, pos, box, q, sigma, eps, excl_off, excl_idx, rc, es_mode,
                                  kappa, nthreads, forces, energies, atom_energy);
}

int64_t orc_nonbonded_em(int n, const double* pos, const double* box, const double* q,
                         const double* sigma, const double* eps, const int* excl_off,
                         const int* excl_idx, double rc, int es_mode, double kappa, int nthreads,
                         double* forces, double* energies) {
    return nonbonded_impl<double>(n, pos, box, q, sigma, eps, excl_off, excl_idx, rc, es_mode,
                                  kappa, nthreads, forces, energies, nullptr, true);
}

int64_t orc_pairset(int n, const double* pos, const double* box, const int* excl_off,
                    const int* excl_idx, double rc, double band, int64_t cap, int32_t* pairs,
                    uint8_t* band_flag, int64_t* n_band) {
    CellGrid grid;
    grid.build(n, pos, box, rc + band);
    std::vector<std::pair<int, int>> out;
    std::vector<uint8_t> flags;
    int64_t nb = 0;
    for (int i = 0; i < n; ++i) {
        const D3 pi = load(pos, i);
        auto body = [&](int j) {
            if (j <= i) return;
            if (is_excluded(excl_off, excl_idx, i, j)) return;
            const D3 d = min_image(load(pos, j) - pi, box);
            const double r = len(d);
            const bool in_band = std::fabs(r - rc) < band;
            if (r <= rc || in_band) {
                if (r <= rc) out.push_back({i, j}), flags.push_back(in_band ? 1 : 0);
                if (in_band) ++nb;
            }
        };
        if (grid.ok)
            grid.visit(pos + 3 * i, box, body);
        else
            for (int j = 0; j < n; ++j) body(j);
    }
    std::vector<size_t> order(out.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = k;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return out[a] < out[b]; });
    const int64_t total = (int64_t)out.size();
    for (int64_t k = 0; k < total && k < cap; ++k) {
        pairs[2 * k] = out[order[k]].first;
        pairs[2 * k + 1] = out[order[k]].second;
        if (band_flag) band_flag[k] = flags[order[k]];
    }
    if (n_band) *n_band = nb;
    return total;
}

static void bonded_impl(const double* pos, const double* box, int nb, const int* bidx,
                        const double* bpar, int na, const int* aidx, const double* apar, int nd,
                        const int* didx, const double* dpar, int ni, const int* iidx, const double* ipar,
                        int np, const int* pidx, const double* ppar, double* forces, double* energies,
                        double* atom_energy) {
    // a term's energy is shared equally by its atoms in atom_energy
    auto share = [&](const int* idx, int k, double e) {
        if (atom_energy)
            for (int a = 0; a < k; ++a) atom_energy[idx[a]] += e / k;
    };
    // positions of a term's atoms unwrapped by the minimum image relative to its first atom
    auto gather = [&](const int* idx, int k, D3* p) {
        p[0] = load(pos, idx[0]);
        for (int a = 1; a < k; ++a) p[a] = p[0] + min_image(load(pos, idx[a]) - p[0], box);
    };
    D3 p[4], f[4];
    double e;
    for (int t = 0; t < nb; ++t) {
        gather(bidx + 2 * t, 2, p);
        bond_term(p[0], p[1], bpar[2 * t], bpar[2 * t + 1], f, &e);
        for (int a = 0; a < 2; ++a) addf(forces, bidx[2 * t + a], f[a]);
        energies[0] += e;
        share(bidx + 2 * t, 2, e);
    }
    for (int t = 0; t < na; ++t) {
        gather(aidx + 3 * t, 3, p);
        angle_term(p[0], p[1], p[2], apar + 4 * t, f, &e);
        for (int a = 0; a < 3; ++a) addf(forces, aidx[3 * t + a], f[a]);
        energies[1] += e;
        share(aidx + 3 * t, 3, e);
    }
    for (int t = 0; t < nd; ++t) {
        gather(didx + 4 * t, 4, p);
        dihedral_term(p[0], p[1], p[2], p[3], dpar + 3 * t, f, &e);
        for (int a = 0; a < 4; ++a) addf(forces, didx[4 * t + a], f[a]);
        energies[2] += e;
        share(didx + 4 * t, 4, e);
    }
    for (int t = 0; t < ni; ++t) {
        gather(iidx + 4 * t, 4, p);
        improper_term(p[0], p[1], p[2], p[3], ipar + 2 * t, f, &e);
        for (int a = 0; a < 4; ++a) addf(forces, iidx[4 * t + a], f[a]);
        energies[3] += e;
        share(iidx + 4 * t, 4, e);
    }
    for (int t = 0; t < np; ++t) {
        gather(pidx + 2 * t, 2, p);
        pairbond_term(p[0], p[1], ppar[2 * t], ppar[2 * t + 1], f, &e);
        for (int a = 0; a < 2; ++a) addf(forces, pidx[2 * t + a], f[a]);
        energies[4] += e;
        share(pidx + 2 * t, 2, e);
    }
}

void orc_bonded(int n, const double* pos, const double* box, int nb, const int* bidx,
                const double* bpar, int na, const int* aidx, const double* apar, int nd,
                const int* didx, const double* dpar, int ni, const int* iidx, const double* ipar,
                int np, const int* pidx, const double* ppar, double* forces, double* energies) {
    (void)n;
    bonded_impl(pos, box, nb, bidx, bpar, na, aidx, apar, nd, didx, dpar, ni, iidx, ipar, np, pidx, ppar,
                forces, energies, nullptr);
}

void orc_bonded_atoms(int n, const double* pos, const double* box, int nb, const int* bidx,
                      const double* bpar, int na, const int* aidx, const double* apar, int nd,
                      const int* didx, const double* dpar, int ni, const int* iidx, const double* ipar,
                      int np, const int* pidx, const double* ppar, double* forces, double* energies,
                      double* atom_energy) {
    (void)n;
    bonded_impl(pos, box, nb, bidx, bpar, na, aidx, apar, nd, didx, dpar, ni, iidx, ipar, np, pidx, ppar,
                forces, energies, atom_energy);
}

void orc_pme(int n, const double* pos, const double* q, const double* box, int kx, int ky, int kz,
             double kappa, int influence, int gather, double* forces, double* energies,
             double* potential_out) {
    const int K[3] = {kx, ky, kz};
    const size_t N = (size_t)kx * ky * kz;
    const double V = box[0] * box[1] * box[2];
    std::vector<cd> grid(N, cd(0, 0));
    auto idx = [&](int x, int y, int z) {
        return (size_t)wrapi(x, kx) + (size_t)kx * ((size_t)wrapi(y, ky) + (size_t)ky * wrapi(z, kz));
    };
    // spread Q(m) = sum_j q_j W(u_j - m)   (PME.cuh:249-300 without the 1/h^3 factor)
    std::vector<int> base(3 * (size_t)n);
    std::vector<double> W(12 * (size_t)n), dW(12 * (size_t)n);
    for (int j = 0; j < n; ++j) {
        for (int d = 0; d < 3; ++d) {
            double u = pos[3 * j + d] / box[d] * K[d];
            double fl = std::floor(u);
            double f = u - fl;
            base[3 * j + d] = (int)fl;
            bspline4(f, &W[12 * j + 4 * d], &dW[12 * j + 4 * d]);
        }
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b)
                for (int c = 0; c < 4; ++c)
                    grid[idx(base[3 * j] - 1 + a, base[3 * j + 1] - 1 + b, base[3 * j + 2] - 1 + c)] +=
                        q[j] * W[12 * j + a] * W[12 * j + 4 + b] * W[12 * j + 8 + c];
    }
    fft3d(kx, ky, kz, grid.data(), -1);
    const double pi_c = influence == 1 ? kPiRef : kPi;
    for (int z = 0; z < kz; ++z)
        for (int y = 0; y < ky; ++y)
            for (int x = 0; x < kx; ++x) {
                const int m[3] = {x <= kx / 2 ? x : x - kx, y <= ky / 2 ? y : y - ky, z <= kz / 2 ? z : z - kz};
                double kv[3], k2 = 0;
                for (int d = 0; d < 3; ++d) {
                    kv[d] = 2.0 * pi_c * m[d] / box[d];
                    k2 += kv[d] * kv[d];
                }
                double th = 0.0;
                if (m[0] != 0 || m[1] != 0 || m[2] != 0) {
                    const double g = 4.0 * pi_c / k2 * std::exp(-k2 / (4.0 * kappa * kappa)) * kCoulomb;
                    if (influence == 1) {
                        th = influence_ref(m, box, K, kappa) * (double)N / V;
                    } else {
                        double B = 1.0;
                        for (int d = 0; d < 3; ++d) {
                            const double b = 2.0 / 3.0 + std::cos(2.0 * kPi * m[d] / K[d]) / 3.0;
                            B *= b * b;
                        }
                        th = g / B * (double)N / V;
                    }
                }
                grid[idx(x, y, z)] *= th;
            }
    fft3d(kx, ky, kz, grid.data(), +1);
    // phi(m) = (1/N) IDFT(theta * DFT(Q))
    const double invN = 1.0 / (double)N;
    double e_rec = 0.0;
    for (int j = 0; j < n; ++j) {
        double phi = 0.0;
        D3 grad{0, 0, 0};
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b)
                for (int c = 0; c < 4; ++c) {
                    const int gx = base[3 * j] - 1 + a, gy = base[3 * j + 1] - 1 + b, gz = base[3 * j + 2] - 1 + c;
                    const double wx = W[12 * j + a], wy = W[12 * j + 4 + b], wz = W[12 * j + 8 + c];
                    const double ph = grid[idx(gx, gy, gz)].real() * invN;
                    phi += wx * wy * wz * ph;
                    if (gather == 0) {
                        grad.x += dW[12 * j + a] * kx / box[0] * wy * wz * ph;
                        grad.y += wx * dW[12 * j + 4 + b] * ky / box[1] * wz * ph;
                        grad.z += wx * wy * dW[12 * j + 8 + c] * kz / box[2] * ph;
                    } else {
                        const double w = wx * wy * wz;
                        grad.x += w * (grid[idx(gx + 1, gy, gz)].real() - grid[idx(gx - 1, gy, gz)].real()) * invN * kx / (2.0 * box[0]);
                        grad.y += w * (grid[idx(gx, gy + 1, gz)].real() - grid[idx(gx, gy - 1, gz)].real()) * invN * ky / (2.0 * box[1]);
                        grad.z += w * (grid[idx(gx, gy, gz + 1)].real() - grid[idx(gx, gy, gz - 1)].real()) * invN * kz / (2.0 * box[2]);
                    }
                }
        addf(forces, j, grad * (-q[j]));
        e_rec += 0.5 * q[j] * phi;
        if (potential_out) potential_out[j] = phi;
    }
    double q2 = 0.0;
    for (int j = 0; j < n; ++j) q2 += q[j] * q[j];
    energies[0] += e_rec;
    energies[1] += -kappa / std::sqrt(pi_c) * q2 * kCoulomb;
}

void orc_ewald_recip(int n, const double* pos, const double* q, const double* box, double kappa,
                     int mmax, double* forces, double* energy) {
    const double V = box[0] * box[1] * box[2];
    double e = 0.0;
    std::vector<double> c(n), s(n);
    for (int mx = -mmax; mx <= mmax; ++mx)
        for (int my = -mmax; my <= mmax; ++my)
            for (int mz = -mmax; mz <= mmax; ++mz) {
                if (mx == 0 && my == 0 && mz == 0) continue;
                const double k[3] = {2 * kPi * mx / box[0], 2 * kPi * my / box[1], 2 * kPi * mz / box[2]};
                const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                const double A = 4 * kPi / k2 * std::exp(-k2 / (4 * kappa * kappa));
                if (A < 1e-300) continue;
                double re = 0, im = 0;
                for (int j = 0; j < n; ++j) {
                    const double th = k[0] * pos[3 * j] + k[1] * pos[3 * j + 1] + k[2] * pos[3 * j + 2];
                    c[j] = std::cos(th);
                    s[j] = std::sin(th);
                    re += q[j] * c[j];
                    im += q[j] * s[j];
                }
                e += kCoulomb / (2 * V) * A * (re * re + im * im);
                for (int j = 0; j < n; ++j) {
                    const double g = kCoulomb / V * A * q[j] * (re * s[j] - im * c[j]);
                    forces[3 * j] += g * k[0];
                    forces[3 * j + 1] += g * k[1];
                    forces[3 * j + 2] += g * k[2];
                }
            }
    *energy += e;
}

void orc_exclusion_correction(int n, const double* pos, const double* q, const double* box,
                              int npairs, const int* pairs, double kappa, double* forces,
                              double* energy) {
    orc_exclusion_correction_atoms(n, pos, q, box, npairs, pairs, kappa, forces, energy, nullptr);
}

void orc_exclusion_correction_atoms(int n, const double* pos, const double* q, const double* box,
                                    int npairs, const int* pairs, double kappa, double* forces,
                                    double* energy, double* atom_energy) {
    (void)n;
    double e = 0.0;
    for (int t = 0; t < npairs; ++t) {
        const int i = pairs[2 * t], j = pairs[2 * t + 1];
        const D3 d = min_image(load(pos, i) - load(pos, j), box);  // r_i - r_j
        const double r = len(d);
        const double qq = q[i] * q[j] * kCoulomb;
        const double er = std::erf(kappa * r);
        e += -qq * er / r;
        if (atom_energy) {
            atom_energy[i] += -0.5 * qq * er / r;
            atom_energy[j] += -0.5 * qq * er / r;
        }
        // F_i = -dE/dr_i = qq * d/dr(erf(kr)/r) * d/r ... with E = -qq erf(kr)/r
        const double dedr = -qq * (2.0 * kappa / std::sqrt(kPi) * std::exp(-kappa * kappa * r * r) / r - er / (r * r));
        const D3 fi = d * (-dedr / r);
        addf(forces, i, fi);
        addf(forces, j, fi * -1.0);
    }
    *energy += e;
}

void orc_integrate(int n, double* pos, double* vel, double* fprev, const double* forces,
                   const double* mass, double dt, int integrator, double scale) {
    for (int i = 0; i < n; ++i) {
        const double im = 1.0 / mass[i];
        for (int d = 0; d < 3; ++d) {
            const int k = 3 * i + d;
            if (integrator == 0) {
                vel[k] = (vel[k] + forces[k] * im * dt) * scale;
                pos[k] += vel[k] * dt;
            } else {
                const double v = vel[k] + (forces[k] + fprev[k]) * dt * 0.5 * im;
                pos[k] += v * dt + forces[k] * 0.5 * im * dt * dt;
                fprev[k] = forces[k];
                vel[k] = v * scale;
            }
        }
    }
}

void orc_em_step(int n, double* pos, const double* forces, double* adam, int step) {
    for (int i = 0; i < n; ++i) {
        double f[3];
        force_activation(&forces[3 * i], 1.0, f);
        adam_move(f, adam + 6 * i, adam + 6 * i + 3, step, &pos[3 * i]);
    }
}

// ------------------------------------------------ per-term entry points
// Each evaluates, sample by sample, the same internal function the system
// loops above use, so that the golden vectors of the reference's own device
// functions pin exactly the code the system-level checks run.

void orc_pair_terms(int n, const double* diff, const double* sig, const double* eps, const double* qq,
                    int es_mode, double kappa, int precision, int em, double* f_out, double* e_out) {
    for (int t = 0; t < n; ++t) {
        if (precision == 32) {
            const V3<float> d{(float)diff[3 * t], (float)diff[3 * t + 1], (float)diff[3 * t + 2]};
            const PairOut<float> o = pair_interaction<float>(d, dot(d, d), (float)sig[t], (float)eps[t], (float)qq[t],
                                                             es_mode, (float)kappa, (float)kCoulomb, (float)kPiRef,
                                                             em != 0);
            f_out[3 * t] = o.f_on_i.x, f_out[3 * t + 1] = o.f_on_i.y, f_out[3 * t + 2] = o.f_on_i.z;
            e_out[2 * t] = o.e_lj, e_out[2 * t + 1] = o.e_coul;
        } else {
            const D3 d = load(diff, t);
            const PairOut<double> o = pair_interaction<double>(d, dot(d, d), sig[t], eps[t], qq[t], es_mode, kappa,
                                                               kCoulomb, kPi, em != 0);
            f_out[3 * t] = o.f_on_i.x, f_out[3 * t + 1] = o.f_on_i.y, f_out[3 * t + 2] = o.f_on_i.z;
            e_out[2 * t] = o.e_lj, e_out[2 * t + 1] = o.e_coul;
        }
    }
}

void orc_bonded_terms(int kind, int n, const double* pos, const double* par, double* f_out, double* e_out) {
    static const int natoms[5] = {2, 3, 4, 4, 2}, npar[5] = {2, 4, 3, 2, 2};
    if (kind < 0 || kind > 4) return;
    const int na = natoms[kind], np = npar[kind];
    for (int t = 0; t < n; ++t) {
        const double* x = pos + (size_t)3 * na * t;
        const double* p = par + (size_t)np * t;
        D3 f[4];
        double e = 0.0;
        if (kind == 0) bond_term(load(x, 0), load(x, 1), p[0], p[1], f, &e);
        else if (kind == 1) angle_term(load(x, 0), load(x, 1), load(x, 2), p, f, &e);
        else if (kind == 2) dihedral_term(load(x, 0), load(x, 1), load(x, 2), load(x, 3), p, f, &e);
        else if (kind == 3) improper_term(load(x, 0), load(x, 1), load(x, 2), load(x, 3), p, f, &e);
        else pairbond_term(load(x, 0), load(x, 1), p[0], p[1], f, &e);
        for (int a = 0; a < na; ++a) {
            double* o = f_out + (size_t)3 * (na * t + a);
            o[0] = f[a].x, o[1] = f[a].y, o[2] = f[a].z;
        }
        e_out[t] = e;
    }
}

void orc_bspline4(int n, const double* f, double* w) {
    for (int t = 0; t < n; ++t) bspline4(f[t], w + 4 * t, nullptr);
}

void orc_ref_green(int K, double L, double kappa, double* out) {
    // the reference's layout: x (the half dimension, K/2 + 1) fastest, then y, z
    const int H = K / 2 + 1;
    const double box[3] = {L, L, L};
    const int Ks[3] = {K, K, K};
    for (int z = 0; z < K; ++z)
        for (int y = 0; y < K; ++y)
            for (int x = 0; x < H; ++x) {
                const int m[3] = {x, y <= K / 2 ? y : y - K, z <= K / 2 ? z : z - K};
                out[(size_t)x + (size_t)H * ((size_t)y + (size_t)K * z)] = influence_ref(m, box, Ks, kappa);
            }
}

void orc_force_activation(int n, const double* f, double scalar, double* out) {
    for (int t = 0; t < n; ++t) force_activation(f + 3 * t, scalar, out + 3 * t);
}

void orc_adam(int n, const double* f, double* m1, double* m2, const int* step, double* dpos) {
    for (int t = 0; t < n; ++t) {
        dpos[3 * t] = dpos[3 * t + 1] = dpos[3 * t + 2] = 0.0;
        adam_move(f + 3 * t, m1 + 3 * t, m2 + 3 * t, step[t], dpos + 3 * t);
    }
}

int orc_compounds_interact(int n, const double* keys_left, const double* keys_right, const double* radii_left,
                           const double* radii_right, double box_nm, double cutoff, uint8_t* out) {
    int hits = 0;
    for (int t = 0; t < n; ++t) {
        out[t] = compounds_interact(keys_left + 6 * t, keys_right + 6 * t, radii_left + 2 * t,
                                    radii_right + 2 * t, (float)box_nm, (float)cutoff)
                     ? 1
                     : 0;
        hits += out[t];
    }
    return hits;
}

void orc_fft3d(int kx, int ky, int kz, double* data, int sign) {
    fft3d(kx, ky, kz, reinterpret_cast<cd*>(data), sign);
}

void orc_mlp_forward(int rows, const double* x, const double* params, double* y) {
    const int K[4] = {80, 128, 128, 128}, N[4] = {128, 128, 128, 8};
    const double* W[4];
    const double* b[4];
    size_t off = 0;
    for (int l = 0; l < 4; ++l) {
        W[l] = params + off;
        off += (size_t)K[l] * N[l];
        b[l] = params + off;
        off += N[l];
    }
    std::vector<double> a(128), z(128);
    for (int r = 0; r < rows; ++r) {
        std::fill(a.begin(), a.end(), 0.0);
        for (int k = 0; k < 68; ++k) a[k] = x[(size_t)r * 68 + k];
        for (int l = 0; l < 3; ++l) {
            for (int n = 0; n < N[l]; ++n) {
                double s = b[l][n];
                for (int k = 0; k < K[l]; ++k) s += a[k] * W[l][(size_t)k * N[l] + n];
                z[n] = s / (1.0 + std::exp(-s));
            }
            std::copy(z.begin(), z.end(), a.begin());
        }
        for (int n = 0; n < 3; ++n) {
            double s = b[3][n];
            for (int k = 0; k < 128; ++k) s += a[k] * W[3][(size_t)k * 8 + n];
            y[(size_t)r * 3 + n] = s;
        }
    }
}

double orc_mlp_grads(int rows, const double* x, const double* t, const double* params, double* grads) {
    const int K[4] = {80, 128, 128, 128}, N[4] = {128, 128, 128, 8}, nin = 68, nout = 3;
    const double* W[4];
    const double* b[4];
    double* gW[4];
    double* gb[4];
    size_t off = 0;
    for (int l = 0; l < 4; ++l) {
        W[l] = params + off;
        gW[l] = grads + off;
        off += (size_t)K[l] * N[l];
        b[l] = params + off;
        gb[l] = grads + off;
        off += N[l];
    }
    std::fill(grads, grads + off, 0.0);
    double loss = 0.0;
    std::vector<double> a[4], z[3], dz(128), dprev(128);
    for (int l = 0; l < 4; ++l) a[l].assign(128, 0.0);
    for (int l = 0; l < 3; ++l) z[l].assign(128, 0.0);
    std::vector<double> y(8);
    const double inv = 2.0 / (3.0 * rows);
    for (int r = 0; r < rows; ++r) {
        std::fill(a[0].begin(), a[0].end(), 0.0);
        for (int k = 0; k < nin; ++k) a[0][k] = x[(size_t)r * nin + k];
        for (int l = 0; l < 3; ++l) {
            for (int n = 0; n < N[l]; ++n) {
                double s = b[l][n];
                for (int k = 0; k < K[l]; ++k) s += a[l][k] * W[l][(size_t)k * N[l] + n];
                z[l][n] = s;
                a[l + 1][n] = s / (1.0 + std::exp(-s));
            }
        }
        for (int n = 0; n < nout; ++n) {
            double s = b[3][n];
            for (int k = 0; k < 128; ++k) s += a[3][k] * W[3][(size_t)k * 8 + n];
            y[n] = s;
        }
        // backward
        std::fill(dz.begin(), dz.end(), 0.0);
        for (int n = 0; n < nout; ++n) {
            const double e = y[n] - t[(size_t)r * nout + n];
            loss += e * e;
            dz[n] = e * inv;
        }
        for (int n = 0; n < nout; ++n) {
            gb[3][n] += dz[n];
            for (int k = 0; k < 128; ++k) gW[3][(size_t)k * 8 + n] += a[3][k] * dz[n];
        }
        for (int k = 0; k < 128; ++k) {
            double s = 0.0;
            for (int n = 0; n < nout; ++n) s += W[3][(size_t)k * 8 + n] * dz[n];
            dprev[k] = s;
        }
        for (int l = 2; l >= 0; --l) {
            for (int n = 0; n < N[l]; ++n) {
                const double sg = 1.0 / (1.0 + std::exp(-z[l][n]));
                dz[n] = dprev[n] * sg * (1.0 + z[l][n] * (1.0 - sg));
            }
            for (int n = 0; n < N[l]; ++n) {
                gb[l][n] += dz[n];
                for (int k = 0; k < K[l]; ++k) gW[l][(size_t)k * N[l] + n] += a[l][k] * dz[n];
            }
            if (l > 0)
                for (int k = 0; k < K[l]; ++k) {
                    double s = 0.0;
                    for (int n = 0; n < N[l]; ++n) s += W[l][(size_t)k * N[l] + n] * dz[n];
                    dprev[k] = s;
                }
        }
    }
    return loss / (3.0 * rows);
}

}  // extern "C"
