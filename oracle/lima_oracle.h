/*
 * lima_oracle.h — CPU restatement of LIMA's per-step force and integration
 * formulas.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and
 * the CPU-baseline leg of the benchmark call this library as the checker; the
 * product path (liblima_b200.so) never links or calls it.
 *
 * Parity status: the reference ships no golden force vectors (its fixtures
 * live in an external LIMA_data directory that is not distributed).  The
 * oracle is pinned by the reference's own analytic known-answer tests, restated
 * in tests/test_oracle_kat.py:
 *   code/LIMA_TESTS/src/ForceCorrectness.h:115-165  (single bond, 1e-4)
 *   code/LIMA_TESTS/src/ForceCorrectness.h:232-333  (angle + Urey-Bradley, 1e-4)
 *   code/LIMA_TESTS/src/ForceCorrectness.h:336-403  (pair-bond LJ, 1e-4)
 *   code/LIMA_TESTS/src/ElectrostaticsTests.h:19-26 (Coulomb constant, 1e-4)
 *   code/LIMA_TESTS/src/ElectrostaticsTests.h:300-396 (two-particle PME, 7 %)
 *   code/LIMA_TESTS/src/ElectrostaticsTests.h:521-609 (many-ion PME, 18 % mean)
 * plus finite-difference energy/force consistency and an independent Ewald sum.
 *
 * Units are the reference's: nm, ns, kg/mol, kC/mol, J/mol, J/mol/nm.
 * Positions are double[3n], forces are ACCUMULATED into double[3n].
 */
#ifndef LIMA_ORACLE_H
#define LIMA_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

double orc_coulomb_constant(void);       /* k_e in J nm / mol / (kC/mol)^2 */
double orc_e_to_kcmol(void);             /* elementary charge in kC/mol     */

/* Short-range non-bonded forces over all atom pairs (i<j) that are not
 * excluded and whose minimum-image distance r satisfies r <= rc.
 *   LJ (LennardJonesInteractions.cuh:74-108): F_i = 24 eps s(1-2s)/r^2 (r_j-r_i),
 *       s=(sigma/r)^6, E = 4 eps s(s-1); sigma=(s_i+s_j)/2, eps=sqrt(e_i e_j)
 *   Coulomb (DeviceAlgorithmsPrivate.cuh:38-95): es_mode 1 plain k q q/r,
 *       es_mode 2 erfc(kappa r) screened with the matching force term.
 * excl_off[n+1]/excl_idx: CSR list of excluded partners (both directions).
 * precision: 64 = FP64, 32 = FP32 reference-faithful arithmetic.
 * nthreads: OpenMP threads (0 = all).  energies[0]=LJ, [1]=Coulomb,
 * [2]=virial (-1/2 sum r_ij.f_ij).  Returns the number of pairs evaluated. */
int64_t orc_nonbonded(int n, const double* pos, const double* box,
                      const double* q, const double* sigma, const double* eps,
                      const int* excl_off, const int* excl_idx,
                      double rc, int es_mode, double kappa, int precision, int nthreads,
                      double* forces, double* energies);

/* orc_nonbonded in FP64 with the energy-minimisation variant of the LJ pair
 * force: bounded by +-1e20 and passed through the tanh activation with scale
 * 100 (LennardJonesInteractions.cuh:85-101, EngineUtils.cuh:112-140); Coulomb
 * and the energies are unchanged. */
int64_t orc_nonbonded_em(int n, const double* pos, const double* box,
                         const double* q, const double* sigma, const double* eps,
                         const int* excl_off, const int* excl_idx,
                         double rc, int es_mode, double kappa, int nthreads,
                         double* forces, double* energies);

/* orc_nonbonded in FP64 that also adds, per atom, half of the energy of each of
 * its pairs (LJ + Coulomb) to atom_energy[n]: the per-particle potential
 * energy the reference logs (LennardJonesInteractions.cuh:101, factor 0.5). */
int64_t orc_nonbonded_atoms(int n, const double* pos, const double* box,
                            const double* q, const double* sigma, const double* eps,
                            const int* excl_off, const int* excl_idx,
                            double rc, int es_mode, double kappa, int nthreads,
                            double* forces, double* energies, double* atom_energy);

/* Sorted list of pairs (i<j) with r <= rc that are not excluded.  Pairs with
 * |r - rc| < band are counted in *n_band and flagged in band_flag (may be
 * NULL).  Returns the pair count (writes at most cap pairs). */
int64_t orc_pairset(int n, const double* pos, const double* box,
                    const int* excl_off, const int* excl_idx, double rc, double band,
                    int64_t cap, int32_t* pairs, uint8_t* band_flag, int64_t* n_band);

/* Bonded terms, restating code/LIMA_ENGINE/src/ForceComputations.cuh:
 *   bonds      :17-51   params [b0, kb]
 *   angles     :53-115  params [theta0, ktheta, ub0, kub] (Urey-Bradley on)
 *   dihedrals  :119-210 params [phi0, kphi, n]
 *   impropers  :214-264 params [psi0, kpsi]
 *   pair bonds :335-376 params [sigma, eps]
 * Vectors between the atoms of one term use the minimum image (box may be
 * NULL for no periodicity).  energies[0..4] = bond, angle, dihedral, improper,
 * pairbond. */
void orc_bonded(int n, const double* pos, const double* box,
                int nb, const int* bidx, const double* bpar,
                int na, const int* aidx, const double* apar,
                int nd, const int* didx, const double* dpar,
                int ni, const int* iidx, const double* ipar,
                int np, const int* pidx, const double* ppar,
                double* forces, double* energies);

/* orc_bonded that also shares each term's energy equally among its atoms in
 * atom_energy[n]. */
void orc_bonded_atoms(int n, const double* pos, const double* box,
                      int nb, const int* bidx, const double* bpar,
                      int na, const int* aidx, const double* apar,
                      int nd, const int* didx, const double* dpar,
                      int ni, const int* iidx, const double* ipar,
                      int np, const int* pidx, const double* ppar,
                      double* forces, double* energies, double* atom_energy);

/* Smooth PME reciprocal part on a Kx x Ky x Kz grid, order 4, weights placed
 * at floor(u)-1 .. floor(u)+2 as in PME.cuh:249-300 and 335-383.
 * influence 0: SPME  theta(k) = (N/V) k_e 4pi/k^2 exp(-k^2/4kappa^2) / B(k),
 *              B = prod_d (2/3 + 1/3 cos(2 pi m_d/K_d))^2
 * influence 1: the reference's function (PME.cuh:434-495):
 *              (1/h^3) k_e 4pi/k^2 exp(-k^2/4kappa^2) prod_d sinc^8(k_d h_d/2),
 *              with pi truncated to 3.14159 (Constants.h:51)
 * gather 0: analytic B-spline derivative; 1: central difference of the
 *           gridded potential (PME.cuh:384-407).
 * energies[0] = 1/2 sum_j q_j phi(r_j); energies[1] = self term
 * -kappa/sqrt(pi) k_e sum q^2.  potential_out (may be NULL) receives
 * phi(r_j) per atom. */
void orc_pme(int n, const double* pos, const double* q, const double* box,
             int kx, int ky, int kz, double kappa, int influence, int gather,
             double* forces, double* energies, double* potential_out);

/* Reciprocal Ewald sum over all k != 0 with |m_d| <= mmax (FP64). */
void orc_ewald_recip(int n, const double* pos, const double* q, const double* box,
                     double kappa, int mmax, double* forces, double* energy);

/* Reciprocal-space exclusion correction for excluded pairs (i<j):
 * E = -k_e q_i q_j erf(kappa r)/r with its force. */
void orc_exclusion_correction(int n, const double* pos, const double* q, const double* box,
                              int npairs, const int* pairs, double kappa,
                              double* forces, double* energy);

/* orc_exclusion_correction that also gives half of each pair's energy to
 * each of its atoms in atom_energy[n] (may be NULL). */
void orc_exclusion_correction_atoms(int n, const double* pos, const double* q, const double* box,
                                    int npairs, const int* pairs, double kappa,
                                    double* forces, double* energy, double* atom_energy);

/* One integration step. integrator 0: leapfrog (v(t+dt/2) = v(t-dt/2) + F dt/m;
 * x += v dt); 1: the reference's velocity Verlet (EngineUtils.cuh:31-41,
 * EngineKernels.cuh:399-413): v = v_prev + (F + F_prev) dt/2m,
 * x += v dt + F dt^2/2m, then F_prev = F, v_prev = v * scale.
 * fprev may be NULL for leapfrog. */
void orc_integrate(int n, double* pos, double* vel, double* fprev, const double* forces,
                   const double* mass, double dt, int integrator, double thermostat_scale);

/* One energy-minimisation step (EngineUtils.cuh:44-72 and 112-140): tanh
 * force clamp at 1e6 J/mol/nm, then ADAM with alpha 8000 on forces x 1e-8.
 * adam[6n] = first and second moments; step counts from 1. */
void orc_em_step(int n, double* pos, const double* forces, double* adam, int step);

/* ---- per-term entry points: each runs, sample by sample, the same internal
 * function the system-level calls above use (checked against golden vectors of
 * the reference's own device functions, tests/golden/). */

/* Pair term (LennardJonesInteractions.cuh:74-108, DeviceAlgorithmsPrivate.cuh:38-95):
 * diff[3n] = r_j - r_i, combined sigma/epsilon, qq = q_i q_j [kC/mol]^2; force on i
 * [J/mol/nm] -> f_out[3n]; full pair energies (LJ, Coulomb) -> e_out[2n].
 * precision 32 = the FP32 reference-faithful arithmetic; em = EM clamp variant. */
void orc_pair_terms(int n, const double* diff, const double* sig, const double* eps, const double* qq,
                    int es_mode, double kappa, int precision, int em, double* f_out, double* e_out);
/* Bonded term of one kind per call: 0 bond (2 atoms; b0, kb), 1 angle + UB (3; theta0,
 * k_theta, ub0, k_ub), 2 dihedral (4; phi0, k_phi, n), 3 improper (4; psi0, k_psi),
 * 4 pair bond (2; sigma, epsilon).  pos[3 natoms n], par[npar n]; forces per atom
 * -> f_out[3 natoms n], energy -> e_out[n]. */
void orc_bonded_terms(int kind, int n, const double* pos, const double* par, double* f_out, double* e_out);
/* Order-4 cardinal B-spline weights at fractions f (DeviceAlgorithmsPrivate.cuh:7-30). */
void orc_bspline4(int n, const double* f, double* w);
/* The reference convention's influence function on a K^3 grid of a cubic box L
 * (PME.cuh:434-495), in its half-complex layout (x in 0..K/2 fastest, then y, z). */
void orc_ref_green(int K, double L, double kappa, double* out);
/* Energy-minimisation force activation (EngineUtils.cuh:112-140), scale A = 1e6 scalar. */
void orc_force_activation(int n, const double* f, double scalar, double* out);
/* One ADAM move per sample (EngineUtils.cuh:44-72): updates m1[3n], m2[3n] in place and
 * writes the position change [nm] to dpos[3n]; step[n] counts from 1. */
void orc_adam(int n, const double* f, double* m1, double* m2, const int* step, double* dpos);
/* The reference's compound-neighbour test (Neighborlists.cuh:64-79): two compounds with
 * two key particles each (keys[6n], positions in nm) and their radii[2n] interact when
 * a key pair is closer than cutoff + r_left + r_right, distances in FP32 under the
 * reference's hyper-position rule in a cubic box of box_nm.  out[n] = 0/1; returns the count. */
int orc_compounds_interact(int n, const double* keys_left, const double* keys_right, const double* radii_left,
                           const double* radii_right, double box_nm, double cutoff, uint8_t* out);

/* 3-D complex DFT in FP64 (x fastest), sign -1 forward, +1 inverse (no
 * normalisation).  data is interleaved re,im. */
void orc_fft3d(int kx, int ky, int kz, double* data, int sign);

/* FP64 forward and backward pass of the learned-PME network (no reference
 * counterpart; the checker of the BF16 tensor-core training kernels).
 * Network 68 -> 128 -> 128 -> 128 -> 3, SiLU after each hidden layer.
 * params/grads layout: W1[80][128] b1[128] W2[128][128] b2[128] W3[128][128]
 * b3[128] W4[128][8] b4[8] (W[k][n] maps input k to output n; rows 68..79 of
 * W1 and columns 3..7 of W4 are unused).  x[rows][68], t[rows][3].
 * Loss = mean over rows x 3 of (y - t)^2; returns the loss and overwrites
 * grads with d loss / d params. */
double orc_mlp_grads(int rows, const double* x, const double* t, const double* params, double* grads);

/* FP64 forward pass of the same network: y[rows][3] from normalised inputs x[rows][68]. */
void orc_mlp_forward(int rows, const double* x, const double* params, double* y);

#ifdef __cplusplus
}
#endif
#endif
