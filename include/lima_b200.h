/*
 * lima_b200.h — C-ABI of the B200-native force and integration path.
 *
 * This boundary replaces the per-step path of LIMA_ENGINE's `class Engine`
 * (code/LIMA_ENGINE/include/Engine.cuh:78-170) together with the parts of
 * `Simulation` / `Box` / `SimParams` it consumes
 * (code/LIMA_BASE/include/Simulation.cuh:17-205).  The lifecycle mirrors the
 * reference:
 *
 *   reference                                         this library
 *   ------------------------------------------------  -----------------------------------
 *   Engine::Engine(unique_ptr<Simulation>, bc, log)    lima_create / lima_create_batch
 *     (code/LIMA_ENGINE/src/Engine.cu:19-81)             + lima_set_box / lima_set_atoms /
 *   BoxBuilder::BuildBox, buildMolecules                  lima_set_bonds ... / lima_set_state
 *     (code/LIMA_MD/src/Environment.cpp:52-67)
 *   SimParams (Simulation.cuh:17-46)                   lima_params
 *   Engine::step()            (Engine.cu:148-159)      lima_step(h, 1)
 *   Environment::run loop     (Environment.cpp:182-230) lima_step(h, n_steps)
 *   em_variant=true run       (Programs.cpp:155-200)   lima_minimize
 *   Engine::takeBackSim()     (EngineHostside.h:10-14) lima_get_state / lima_get_forces
 *   Engine::~Engine           (Engine.cu:83-101)       lima_destroy
 *   SimSignals::critical_error_encountered             lima_get_status (device status word)
 *     (Simulation.cuh:48-50)
 *   runtime_error from genericErrorCheck               every call returns a LIMA_ERR_* code;
 *     (code/LIMA_BASE/include/Utilities.h:22-51)         lima_last_error gives the message
 *
 * Units are the reference's own (code/LIMA_BASE/include/Constants.h:43-60):
 * length nm, time ns, mass kg/mol, charge kC/mol (e x 96.485), energy J/mol,
 * force J/mol/nm.  LJ sigma in nm, epsilon in J/mol; bond k in J/mol/nm^2;
 * angle k in J/mol/rad^2; dihedral k_phi in J/mol (used as given: the
 * reference halves the file value at load, code/LIMA_BASE/src/Bodies.cpp:36-38,
 * and a caller passing reference-loaded parameters passes the halved value).
 *
 * Ownership: every array argument is caller-owned host memory that is copied
 * during the call; nothing retains caller pointers.  Calls on one handle are
 * not thread-safe; distinct handles are independent.
 */
#ifndef LIMA_B200_H
#define LIMA_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define LIMA_API __attribute__((visibility("default")))
#else
#define LIMA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- errors */
#define LIMA_OK                 0
#define LIMA_ERR_INVALID_ARG    1  /* bad pointer, size or parameter              */
#define LIMA_ERR_CUDA           2  /* a CUDA runtime call failed                   */
#define LIMA_ERR_STATE          3  /* call made in the wrong lifecycle state       */
#define LIMA_ERR_OVERFLOW       4  /* a fixed-capacity device list overflowed      */
#define LIMA_ERR_TIMEOUT        5  /* a bounded device wait gave up                */
#define LIMA_ERR_NO_DEVICE      6  /* no CUDA device / wrong architecture          */
#define LIMA_ERR_NOT_FINITE     7  /* NaN or Inf met in positions or forces        */
#define LIMA_ERR_UNSUPPORTED    8  /* option not available in this build           */

/* device status word bits (lima_get_status); mirrors SimSignals plus the
 * overflow checks of Neighborlists.cuh:184-186,214-217,274-276 */
#define LIMA_STATUS_PAIRLIST_OVERFLOW  0x1u
#define LIMA_STATUS_COLUMN_OVERFLOW    0x2u
#define LIMA_STATUS_NONFINITE          0x4u
/* a force accumulator reached half the int64 fixed-point range (2^30 J/mol/nm):
   overlapping atoms; the forces of that step are not trustworthy */
#define LIMA_STATUS_FORCE_SATURATED    0x8u
/* an atom moved more than half the Verlet buffer (skin) since the pair list was
   built: pairs that came within the cutoff may be missing until the next build */
#define LIMA_STATUS_MOVED_TOO_FAR      0x10u
#define LIMA_STATUS_MLP_FALLBACK       0x20u

/* ---------------------------------------------------------------- options */
#define LIMA_ES_NONE    0  /* no electrostatics                               */
#define LIMA_ES_CUTOFF  1  /* plain 1/r Coulomb truncated at the cutoff         */
#define LIMA_ES_EWALD   2  /* erfc real space (+ PME when a PME grid is given)  */

#define LIMA_INTEGRATOR_LEAPFROG 0
#define LIMA_INTEGRATOR_VV       1  /* the reference's velocity-Verlet ("VVS")
                                       code/LIMA_ENGINE/src/EngineUtils.cuh:31-41 */

#define LIMA_CALC_FORCES   0x0
#define LIMA_CALC_ENERGY   0x1

typedef struct lima_params {
    int    device;            /* CUDA device ordinal                                 */
    double dt;                /* [ns]  (reference SimParams::dt)                      */
    double cutoff;            /* [nm]  (SimParams::cutoff_nm)                         */
    double skin;              /* [nm]  Verlet buffer of the cluster pair list; <0: auto */
    int    nstlist;           /* steps between pair-list rebuilds                     */
    int    electrostatics;    /* LIMA_ES_*                                            */
    int    pme_grid[3];       /* default PME grid for every system; 0 = none          */
    double pme_spacing;       /* [nm] if >0 and pme_grid is 0, grid from spacing      */
    double ewald_kappa;       /* [1/nm]; 0 = derive (ewald_tol, or 3/rc in ref_compat) */
    double ewald_tol;         /* erfc(kappa*rc) target when kappa is derived          */
    int    ref_compat;        /* 1 = the reference's reciprocal-space conventions:
                                 kappa = 3/rc (PhysicsUtils.cuh:60-62), influence
                                 function x sinc^8 (PME.cuh:434-495), central-difference
                                 gather (PME.cuh:384-407), no exclusion correction,
                                 self energy added per charged atom (PME.cuh:417-420) */
    int    integrator;        /* LIMA_INTEGRATOR_*                                    */
    double thermostat_scalar; /* velocity scale applied each step (1 = NVE)           */
    int    exclude_bonded;    /* 1 = every atom pair sharing a bond, angle, dihedral
                                 or improper is excluded from LJ and Coulomb
                                 (code/LIMA_TOOLS/src/CompoundBuilder.cpp:40-60)      */
    int    use_graphs;        /* G > 0: replay each block of G pair-list periods (a rebuild and
                                 nstlist steps each) as one CUDA graph; 0 = launch eagerly */
    /* thermostat (code/LIMA_ENGINE/src/Thermostat.cuh:55-103, Engine.cu:167-174): every
       thermostat_interval steps the temperature of each system is measured from its
       kinetic energy (3N - 3 degrees of freedom); with apply_thermostat the integrator's
       velocity scale becomes clamp(target/T, 1 -+ 0.001/thermostat_interval) */
    int    apply_thermostat;  /* 0 = measure only                                      */
    int    thermostat_interval; /* steps between measurements; 0 = never (default 200) */
    double target_temperature; /* [K] (the reference's fixed 310 K)                    */
    /* per-particle logging (EngineUtils.cuh:143-158, Engine.cu:203-240): every
       log_interval steps (0 = off) the position, potential energy, force and speed of
       every atom go to a device ring of log_ring frames, offloaded to host memory
       whenever it fills; read with lima_get_log.  As in the reference
       (EngineKernels.cuh:399-433) a frame is taken after the step's update: the new
       position, the energy and force evaluated at the old one, the updated speed */
    int    log_interval;
    int    log_ring;          /* frames held on the device (default 5, as the reference) */
    /* boundary condition (BoundaryConditionSelect, code/LIMA_BASE/include/Simulation.cuh:13;
       BoundaryCondition.cuh): 1 = periodic (PBC, default); 0 = none (NoBC): no images,
       no wrapping of positions, plain differences in every term; the box only sets the
       column grid (atoms outside it are binned at its edge); needs cutoff Coulomb or none */
    int    periodic;
    /* dynamic pruning (no counterpart in the reference, whose list has no buffer):
       every prune_interval steps, starting at each rebuild, the pair list is cut to
       the rows within an inner radius rc + skin * prune_interval / nstlist of the
       current positions, and the pair kernel walks that shorter list until the
       next prune; 0 = off; < 0 = auto (every 2 steps for an engine of one system with
       at least 1,024 8-atom clusters and nstlist >= 4, else off) */
    int    prune_interval;
    /* warps per i-cluster in the pair kernel and the pair-list search (no
       counterpart in the reference): 1, 2, 4 or 8 (a value in between is rounded
       down) splits every system's rows, and its search window, over that many warps; < 0 = auto (an engine of one system splits so
       that it has up to ~4,096 pair-kernel warps: 8 for 3,000 atoms, 1 from ~16,400;
       a batch does not split); 0 = 1.  Results depend on the split (FP32 sums
       per part), so a system gives the same bits alone and inside a batch when
       both use the same explicit split */
    int    pair_split;
} lima_params;

typedef struct lima_energies {
    double lj;                /* short-range Lennard-Jones                 [J/mol] */
    double coulomb_real;      /* cutoff or erfc real-space Coulomb         [J/mol] */
    double pme_recip;         /* reciprocal-space energy                   [J/mol] */
    double pme_self;          /* Ewald self term                           [J/mol] */
    double pme_excl;          /* reciprocal exclusion correction           [J/mol] */
    double bond, angle, dihedral, improper, pairbond;             /*        [J/mol] */
    double kinetic;           /*                                           [J/mol] */
    double potential;         /* sum of the potential terms                [J/mol] */
    double total;             /* potential + kinetic                       [J/mol] */
    double virial;            /* -1/2 sum r_ij . f_ij (short-range + bonded) [J/mol] */
    double temperature;       /* [K], dof = 3N - 3                                  */
    int64_t step;
} lima_energies;

typedef struct lima_timings {   /* averages over the steps since the last reset [us] */
    double nblist;            /* pair-list rebuild, per rebuild                        */
    double nonbonded, bonded, pme, integrate;  /* per step; 0 unless phase timing is on */
    double step;              /* whole step, device time on the main stream            */
    int64_t steps;
    int64_t rebuilds;
    int64_t kernel_launches;  /* kernels of this library launched since the reset     */
    int32_t pair_shape;       /* launch shape of the force-only pair kernel (lima_autotune) */
    int32_t reserved;
} lima_timings;

typedef struct lima_engine lima_engine;

/* --------------------------------------------------------------- lifecycle */
LIMA_API void        lima_default_params(lima_params* p);
LIMA_API const char* lima_error_string(int code);
LIMA_API const char* lima_last_error(const lima_engine* h);
LIMA_API int         lima_version(void);

/* Engine::Engine (Engine.cu:19-81) for one system. */
LIMA_API int lima_create(const lima_params* p, lima_engine** out);
/* Many independent systems stepped together by the same launches. */
LIMA_API int lima_create_batch(const lima_params* p, int n_systems, lima_engine** out);
/* Engine::~Engine (Engine.cu:83-101). */
LIMA_API int lima_destroy(lima_engine* h);
/* Selects the system that the following set/get calls address (default 0). */
LIMA_API int lima_select_system(lima_engine* h, int system);
LIMA_API int lima_num_systems(const lima_engine* h, int* n);

/* ------------------------------------------------------ box and topology
 * BoxParams::boxSize (Simulation.cuh:55) is an integer cube in the reference;
 * here the box is rectangular with real edge lengths. */
LIMA_API int lima_set_box(lima_engine* h, double lx, double ly, double lz);
/* Per-atom charge [kC/mol], mass [kg/mol], LJ sigma [nm], epsilon [J/mol].
 * Mixing is Lorentz-Berthelot: sigma_ij=(s_i+s_j)/2, eps_ij=sqrt(e_i e_j)
 * (code/LIMA_ENGINE/src/LennardJonesInteractions.cuh:14-27,186-188). */
LIMA_API int lima_set_atoms(lima_engine* h, int n_atoms, const float* charge, const float* mass,
                   const float* sigma, const float* epsilon);
/* SingleBond (Bodies.cuh), params per bond: b0 [nm], kb [J/mol/nm^2]. */
LIMA_API int lima_set_bonds(lima_engine* h, int n, const int32_t* atoms2, const float* params2);
/* AngleUreyBradleyBond, params: theta0 [rad], ktheta, ub0 [nm], kub. */
LIMA_API int lima_set_angles(lima_engine* h, int n, const int32_t* atoms3, const float* params4);
/* DihedralBond, params: phi0 [rad], k_phi [J/mol], multiplicity n. */
LIMA_API int lima_set_dihedrals(lima_engine* h, int n, const int32_t* atoms4, const float* params3);
/* ImproperDihedralBond, params: psi0 [rad], k_psi [J/mol/rad^2]. */
LIMA_API int lima_set_impropers(lima_engine* h, int n, const int32_t* atoms4, const float* params2);
/* PairBond (LJ 1-4 style), params: sigma [nm], epsilon [J/mol]. */
LIMA_API int lima_set_pairbonds(lima_engine* h, int n, const int32_t* atoms2, const float* params2);
/* Extra excluded pairs on top of the bonded-term rule. */
LIMA_API int lima_set_exclusions(lima_engine* h, int n, const int32_t* atoms2);
/* Compound membership, the unit the reference's builder groups atoms into
 * (CompoundBuilder.cpp:425-565; at most 32 atoms per compound, Constants.h:91)
 * and the bonded compound pairs (CreateCompounds, CompoundBuilder.cpp:546-560;
 * at most 6 per compound, Bodies.cuh:205).  compound[n_atoms]: the compound of
 * each atom of the selected system, or -1 for none; bonded[2 n_bonded]:
 * compound ids.  Used with ref_compat = 1: as in the reference's
 * immediate-neighbour kernel (EngineKernels.cuh:150-317 with
 * LennardJonesInteractions.cuh:121-161), every atom pair inside one compound or
 * across two bonded compounds, minus the excluded pairs, is evaluated with no
 * cutoff (LJ and real-space Coulomb), and only all other pairs go through the
 * cutoff pair list.  Without ref_compat the membership is kept but unused. */
LIMA_API int lima_set_compounds(lima_engine* h, int n_atoms, const int32_t* compound, int n_bonded,
                                const int32_t* bonded);
/* Per-system PME grid; overrides lima_params.pme_grid / pme_spacing. */
LIMA_API int lima_set_pme_grid(lima_engine* h, int nx, int ny, int nz);
/* Uniform external electric field [V/nm] on the selected system (default 0):
 * every atom feels q E (q [kC/mol] x E x 1000 = J/mol/nm), included in the forces
 * that lima_get_forces and the log return, with no potential energy term.
 * Replaces Box::uniformElectricField with SimParams::snf_select =
 * HorizontalChargeField (code/LIMA_BASE/include/Bodies.cuh:363-385,
 * code/LIMA_ENGINE/src/EngineKernels.cuh:321-343); the reference's other
 * snf_select kernels (SupernaturalForces.cuh) have empty bodies. */
LIMA_API int lima_set_electric_field(lima_engine* h, double ex, double ey, double ez);

/* -------------------------------------------------------------------- state
 * pos [nm] x 3N (double), vel [nm/ns] x 3N (NULL = zero), for the selected system.
 * A non-finite position is refused with LIMA_ERR_NOT_FINITE and leaves the engine
 * as it was.  On a built engine the atoms keep their slots and the pair list: a
 * state handed back unchanged keeps the list's nstlist cadence; a moved one keeps
 * the list only while every atom stays within half the Verlet buffer of its
 * position at the last list build, else the list is rebuilt before the next
 * forces.  The previous-step force (velocity Verlet) and the minimiser's moments
 * restart at zero, as for a new input. */
LIMA_API int lima_set_state(lima_engine* h, const double* pos, const float* vel);
LIMA_API int lima_get_state(lima_engine* h, double* pos, float* vel);

/* ---------------------------------------------------------------- stepping */
/* Forces at the current positions, no integration. flags: LIMA_CALC_*. */
LIMA_API int lima_compute_forces(lima_engine* h, int flags);
/* n_steps of Engine::step() (Engine.cu:148-159). Energies are evaluated on the
 * last step. */
LIMA_API int lima_step(lima_engine* h, int n_steps);
/* Energy minimisation: the reference's em_variant path (tanh force clamp +
 * ADAM, code/LIMA_ENGINE/src/EngineUtils.cuh:44-140, early stop on max |F|,
 * Engine.cu:275-291). force_tol in J/mol/nm. */
LIMA_API int lima_minimize(lima_engine* h, double force_tol, int max_steps, int* steps_taken,
                  double* max_force);

/* ---------------------------------------------------------------- readback */
LIMA_API int lima_get_forces(lima_engine* h, double* forces);          /* [J/mol/nm] x 3N */
LIMA_API int lima_get_energies(lima_engine* h, lima_energies* e);
/* Ordered atom pairs (i<j, original indices) within the cutoff that the
 * pair kernel evaluates at the current positions.  Writes up to cap pairs
 * into pairs[2*cap] and the total count into *n. */
LIMA_API int lima_get_pairlist(lima_engine* h, int64_t cap, int32_t* pairs, int64_t* n);
/* Size of the cluster pair list over all systems of the handle (no
 * counterpart in the reference, whose compound lists are fixed-size arrays):
 * the rows built at the last rebuild (an i-cluster of 8 atoms and one j-atom
 * in range of at least one of them), the rows the pair kernel walks each step
 * (fewer than the built rows when the list is pruned between rebuilds), the
 * atom pairs it evaluates (two per row for each pair of i-atoms its chunk of 32
 * rows needs) and the pairs among them within
 * the cutoff at the current positions. */
typedef struct lima_pairlist_stats {
    int64_t rows_built;
    int64_t rows_walked;
    int64_t pairs_evaluated;
    int64_t pairs_in_cutoff;
    int64_t reserved[4];
} lima_pairlist_stats;
LIMA_API int lima_get_pairlist_stats(lima_engine* h, lima_pairlist_stats* out);
LIMA_API int lima_get_status(lima_engine* h, uint32_t* status);
LIMA_API int lima_clear_status(lima_engine* h);
LIMA_API int lima_get_timings(lima_engine* h, lima_timings* t);
LIMA_API int lima_reset_timings(lima_engine* h);
/* Times each phase with CUDA events.  While on, the phases run one after the
 * other on one stream (so each measurement covers that phase alone) and every
 * step ends with a device synchronisation. */
LIMA_API int lima_enable_phase_timing(lima_engine* h, int enable);

/* ------------------------------------------------ allocation-free PME stage
 * No counterpart in the reference: this entry point exists for callers that
 * may not allocate device memory: a plug-in inside an application that owns
 * every device allocation through its own pool (a cudaMalloc of its own would
 * bypass the host's accounting and can fail or fragment the pool), or a
 * real-time loop that must not allocate after start-up (cudaMalloc may
 * synchronise the device and take unbounded time).  It computes the smooth-PME reciprocal forces and energy of
 * one set of charges with the engine's own PME kernels (accurate conventions:
 * B-spline moduli, analytic gather), using a static scratch array instead of
 * allocated grids; it calls no allocator.
 *   d_xyzq   device array of n_atoms x {x, y, z [nm], q [kC/mol]} (float)
 *   d_forces device array of n_atoms x 3 doubles, overwritten [J/mol/nm]
 *   d_energy device pointer to one double: 1/2 sum q phi [J/mol] (no self term)
 *   stream   a cudaStream_t, or NULL for the default stream; the call is
 *            asynchronous on it and uses the current device
 * Limits: at most 64^3 real grid points and 128 points per dimension; larger
 * grids return LIMA_ERR_OVERFLOW; dimensions must factor into 2, 3 and 5
 * (LIMA_ERR_UNSUPPORTED otherwise).  Every GPU that loads the library holds
 * about 5 MB of static device memory for it until the process exits.  The first
 * call on a device looks up the scratch array's device address (and looks it up
 * again whenever the device's context has changed, e.g. after cudaDeviceReset);
 * make that first call before any stream capture.  All calls share the array and it
 * keeps the last call's contents (each call clears what must start at zero):
 * calls that overlap on the GPU race. */
LIMA_API int lima_pme_recip_noalloc(const float* d_xyzq, int n_atoms, double lx, double ly, double lz,
                                    int kx, int ky, int kz, double kappa, double* d_forces,
                                    double* d_energy, void* stream);

/* ------------------------------------------------ learned coarse-grid PME
 * No counterpart in the reference (LIMA has no learned component).  A small
 * network (68 -> 128 -> 128 -> 128 -> 3, SiLU, BF16 tensor-core kernels with
 * FP32 accumulation) predicts, per atom, the difference between the full-grid
 * and a coarse-grid PME reciprocal force from the coarse force, the charge and
 * a 64-value descriptor of the charges within 0.8 nm (16 Gaussians x 4
 * channels: q_j, q_j x/r, q_j y/r, q_j z/r, cosine cutoff).  While enabled, the
 * step's reciprocal part is coarse PME + network; the full grid runs every
 * check_interval steps and on every step that evaluates energies, its forces
 * are used on those steps, and once the relative RMSE of the predicted
 * reciprocal force exceeds the tolerance the engine falls back to plain PME
 * for good (until re-enabled).  Requires PME electrostatics and box edges
 * above 1.8 nm.  Calls apply to every system of a batch. */

/* Allocates the coarse grid (each dimension >= 8, factors 2, 3, 5), the
 * network (fixed-seed Glorot-uniform initialisation) and a ring of max_frames
 * training frames. */
LIMA_API int lima_learned_pme_setup(lima_engine* h, int coarse_x, int coarse_y, int coarse_z, int max_frames);
/* Labels the current state: features from the coarse grid, target = full-grid
 * minus coarse-grid reciprocal force.  The first frame fixes the input
 * normalisation and the output scale. */
LIMA_API int lima_learned_pme_collect(lima_engine* h);
/* Adam (beta 0.9/0.999) on the collected frames, rows shuffled per epoch by
 * seed; batch <= 65536 rows.  final_loss (may be NULL): mean squared error of
 * the normalised residual over the last epoch. */
LIMA_API int lima_learned_pme_train(lima_engine* h, int epochs, int batch, float lr, uint64_t seed,
                                    double* final_loss);
/* Turns the correction on or off in stepping; check_interval <= 0 means 50,
 * tolerance <= 0 means 1e-3.  Clears an earlier fallback. */
LIMA_API int lima_learned_pme_enable(lima_engine* h, int on, int check_interval, double tolerance);
/* Relative RMSE of the coarse and of the corrected reciprocal force against
 * the full grid on the current state. */
LIMA_API int lima_learned_pme_eval(lima_engine* h, double* coarse_rel, double* learned_rel);
/* active: the correction is in use; fell_back: a check failed; last_rel: the
 * last check's relative RMSE (-1 before the first check). */
LIMA_API int lima_learned_pme_status(lima_engine* h, int* active, int* fell_back, double* last_rel);
/* Reads (get != 0) or writes the model state: parameters W1[80][128] b1[128]
 * W2[128][128] b2[128] W3[128][128] b3[128] W4[128][8] b4[8] (W[k][n]: input k
 * to output n; rows 68..79 of W1 and columns 3..7 of W4 unused), then the 68
 * input means, the 68 input scales and the output scale.  *needed receives the
 * count (44,561 floats); buf may be NULL to query it. */
LIMA_API int lima_learned_pme_weights(lima_engine* h, int get, float* buf, int64_t n, int64_t* needed);
/* One forward/backward pass without an update on caller rows (x: rows x 68
 * normalised inputs, t: rows x 3 targets, rows <= 65536): grads receives
 * d loss / d parameters in the layout above (44,424 floats), loss the mean
 * squared error.  For checking the training kernels. */
LIMA_API int lima_learned_pme_gradients(lima_engine* h, int rows, const float* x, const float* t,
                                        float* grads, double* loss);
/* Network output for caller rows (features: rows x 68 raw inputs, normalised
 * with the model's statistics inside; out: rows x 3, in units of the output
 * scale), rows <= 65536.  impl 0: the tcgen05 tensor-core kernel used in
 * stepping; 1: the warp-level mma.sync kernel; 2: a self-test of the tcgen05
 * kernel's bounded waits — its first layer's MMAs are withheld, so every wait
 * for them runs out (about a second) and the call returns LIMA_ERR_TIMEOUT with
 * the engine still usable.  LIMA_ERR_TIMEOUT if a bounded device wait gave up. */
LIMA_API int lima_learned_pme_predict(lima_engine* h, int rows, const float* features, float* out, int impl);

/* Autotuner (no counterpart in the reference, whose launch shapes are fixed):
 * after one untimed period per shape, times `periods` pair-list periods of real
 * MD steps (they advance the simulation), three rounds, with each of the 12
 * launch shapes of the pair kernel — 256 or 128 threads per block, with or
 * without leaving SM room to the PME and bonded kernels of the step, one or two
 * pair-list rows' loads in flight per lane, or the persistent kernel whose rows
 * and j-atoms are staged through shared memory — and keeps the fastest for
 * this engine.  All shapes give identical results.  *shape (may be NULL)
 * receives the choice: bit 0 room left, bit 1 128-thread blocks, bit 2 two
 * rows in flight (bit 3 clear), bit 3 the staged persistent kernel. */
LIMA_API int lima_autotune(lima_engine* h, int periods, int* shape);
/* Sets the pair kernel's launch shape (0-11, as lima_autotune reports it). */
LIMA_API int lima_set_pair_shape(lima_engine* h, int shape);

/* ---------------------------------------------------------- thermostat, log */
/* Last temperature measurement of the selected system: temperature [K], the
 * velocity scale in use, and the step it was taken at (-1 before the first). */
LIMA_API int lima_get_thermostat(lima_engine* h, double* temperature, double* scale, int64_t* step);
/* Logged frames of the selected system, oldest first, starting at frame
 * `first`; at most max_frames are written.  Per frame: steps[f] (the step whose
 * forces were evaluated); pos_epot[f][n][4] = x, y, z [nm] after that step's update,
 * potential energy [J/mol] at the step's start (half of each pair energy, an equal
 * share of each bonded term, 1/2 q phi plus the self term); force_speed[f][n][4]
 * = force [J/mol/nm], |v| [nm/ns].  Output arrays may be NULL.  *n_frames
 * receives the number of frames logged so far. */
LIMA_API int lima_get_log(lima_engine* h, int64_t first, int64_t max_frames, int64_t* steps, float* pos_epot,
                          float* force_speed, int64_t* n_frames);
/* Drops every logged frame held on the host. */
LIMA_API int lima_clear_log(lima_engine* h);

#ifdef __cplusplus
}
#endif
#endif /* LIMA_B200_H */
