/* classicalDFT B200 engine: the C ABI of the F[rho] / dF/drho hot path.
 *
 * This is the drop-in boundary behind the reference library's functional API
 * (migduroli/classicalDFT v3.0.0).  The reference has no FFI of its own: its
 * boundary is the C++ call
 *     dft::functionals::total(const physics::Model&, const State&, const Weights&) -> Result
 * (include/dft/functionals/functionals.hpp:64-95) plus the set-up calls that
 * build Weights (functionals.hpp:27-33, fmt/weights.hpp:144-183,
 * functionals/mean_field.hpp:146-219).  Each entry point below names the
 * reference interface it replaces.
 *
 * Conventions (the reference's, functionals.hpp:55-63):
 *   - fields are FP64, N = nx*ny*nz points, flat index iz + nz*(iy + ny*ix);
 *     several species are passed species-major in one array of S*N doubles;
 *   - forces are dOmega/drho * dV (not dOmega/drho);
 *   - chemical potentials are beta*mu (dimensionless), one per species;
 *   - the scalar block is [F, Omega, F_id, F_ext, F_hs, F_mf, N_0 .. N_{S-1}]
 *     with N_s = sum(rho_s) dV, F = F_id + F_ext + F_hs + F_mf and
 *     Omega = F - sum_s mu_s N_s (functionals.hpp:72-92).
 *
 * Every call returns CDFT_OK (0) or a negative status; cdft_last_error()
 * gives the message of the calling thread's last failure.  The C++ host API
 * (include/dft_b200/) rethrows them as std::invalid_argument /
 * std::runtime_error, the reference's exception types.
 *
 * An engine is not thread-safe: use one engine per thread / stream.
 */
#ifndef CDFT_B200_H
#define CDFT_B200_H

#if defined(__GNUC__)
#define CDFT_API __attribute__((visibility("default")))
#else
#define CDFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CDFT_OK 0
#define CDFT_ERR_INVALID (-1) /* std::invalid_argument in the reference */
#define CDFT_ERR_RUNTIME (-2) /* std::runtime_error in the reference */
#define CDFT_ERR_CUDA (-3)
#define CDFT_ERR_CUFFT (-4)

/* FMT models (fmt/models.hpp:153-359, FMTModel::from_name :398-410). */
#define CDFT_ROSENFELD 0
#define CDFT_RSLT 1
#define CDFT_WHITEBEAR_I 2
#define CDFT_WHITEBEAR_II 3
#define CDFT_ESFMT 4

#define CDFT_MAX_SPECIES 4
#define CDFT_MAX_INTERACTIONS 8

/* Precision of the FFTs and k-space products; Phi, dPhi and all sums stay FP64. */
#define CDFT_FP64 0
#define CDFT_MIXED 1

/* Potentials, split schemes and weight schemes
 * (physics/potentials.hpp:18-21, 57-243; physics/interactions.hpp:11-18). */
#define CDFT_POT_LENNARD_JONES 0
#define CDFT_POT_TEN_WOLDE_FRENKEL 1
#define CDFT_POT_WRDF 2
#define CDFT_SPLIT_WCA 0
#define CDFT_SPLIT_BH 1
#define CDFT_WEIGHT_ZERO 0
#define CDFT_WEIGHT_LINEAR_E 1
#define CDFT_WEIGHT_LINEAR_F 2
#define CDFT_WEIGHT_QUADRATIC_F 3
#define CDFT_WEIGHT_GAUSS_E 4
#define CDFT_WEIGHT_GAUSS_F 5

#define CDFT_SCALAR_COUNT 10

typedef struct cdft_engine cdft_engine;

/* A pair potential as built by make_lennard_jones / make_ten_wolde_frenkel /
 * make_wang_ramirez_dobnikar_frenkel (potentials.hpp:311-368). */
typedef struct {
  int type;
  double sigma;
  double epsilon;
  double r_cutoff; /* <= 0: no cutoff (LJ, tWF) */
  double alpha;    /* tWF only */
} cdft_potential;

/* One mean-field interaction (physics/interactions.hpp:23-30 after weight
 * generation): the real-space weight array baked with dV/N, exactly the
 * array the reference FFTs at mean_field.hpp:194. */
typedef struct {
  int species_i;
  int species_j;
  const double* weight_real; /* host, N doubles */
  double a_vdw;
} cdft_interaction;

/* Message of this thread's last failed call ("" if none). */
CDFT_API const char* cdft_last_error(void);

/* One mean-field interaction described by its potential (interactions.hpp:23-30
 * before weight generation): cdft_create_model builds the real-space cell
 * weights and a_vdw on the GPU from it. */
typedef struct {
  int species_i;
  int species_j;
  cdft_potential potential;
  int split;  /* CDFT_SPLIT_* */
  int scheme; /* CDFT_WEIGHT_* */
} cdft_model_interaction;

/* Library version string. */
CDFT_API const char* cdft_version(void);

/* ---- set-up physics (host) ------------------------------------------- */

/* Derived potential parameters: out = {epsilon_shift (WRDF: eps_eff), r_min,
 * v_min, r_zero}.  Replaces make_lennard_jones & co (potentials.hpp:311-368). */
CDFT_API int cdft_potential_info(const cdft_potential* pot, double out[4]);

/* Attractive tail u_att(r) at n radii (potentials.hpp:97-107, 165-175, 228-236). */
CDFT_API int cdft_potential_attractive(const cdft_potential* pot, int split, const double* r, long n, double* out);

/* Barker-Henderson / WCA hard-sphere diameter (potentials.hpp:28-37). */
CDFT_API int cdft_hard_sphere_diameter(const cdft_potential* pot, double kT, int split, double* diameter);

/* (2 pi / kT) int r^2 u_att(r) dr (potentials.hpp:39-50). */
CDFT_API int cdft_vdw_integral(const cdft_potential* pot, double kT, int split, double* value);

/* Real-space mean-field weight w(r)/kT * dV/N on the grid and a_vdw = sum w dV
 * (mean_field.hpp:146-196 up to its FFT).  weight_out: N doubles (host). */
CDFT_API int cdft_interaction_weight(const long shape[3], double dx, const cdft_potential* pot, int split, int scheme,
                            double kT, double* weight_out, double* a_vdw);

/* ---- engine -------------------------------------------------------------- */

/* Build an engine: grid, species diameters, FMT model (esFMT takes A, B) and
 * interactions; uploads and transforms the mean-field weights once.
 * Replaces make_weights(fmt_model, model) (functionals.hpp:27-33) together
 * with the per-call FFTW plans of math/fourier.cpp:25-60.  Runs on the
 * current CUDA device. */
CDFT_API int cdft_create(cdft_engine** out, const long shape[3], double dx, int n_species, const double* diameters,
                int fmt_model, double esfmt_A, double esfmt_B, int n_interactions,
                const cdft_interaction* interactions, int precision);

/* Batched engine: `batch` problems of this grid, species, FMT model and
 * interactions (one mean-field weight set) evaluated together by one set of
 * launches.  cdft_total and cdft_total_device then take every array for all
 * problems back to back: rho, vext and force batch*S*N doubles (problem-
 * major), mu batch*S values and scalars batch*CDFT_SCALAR_COUNT doubles.
 * This is the eval_many of a parameter sweep; problems of different grids
 * use one engine per grid.  No reference counterpart (the reference
 * evaluates one state per call).  The drivers and cdft_hvp need batch 1. */
#define CDFT_MAX_BATCH 64
CDFT_API int cdft_create_batch(cdft_engine** out, const long shape[3], double dx, int n_species,
                               const double* diameters, int fmt_model, double esfmt_A, double esfmt_B,
                               int n_interactions, const cdft_interaction* interactions, int precision, int batch);

/* cdft_create_batch with the mean-field weights made on the GPU: for each
 * interaction the cell weight of mean_field.hpp:42-134 (zero beyond the
 * cut-off plus half a cell diagonal), times dV / N, at every grid offset
 * (mean_field.hpp:146-196), then its FFT; a_vdw = sum of weight * dV
 * (cdft_engine_a_vdw), summed in a fixed order.  The host set-up loop
 * (cdft_interaction_weight) is not run.  kT > 0: the temperature the
 * weights are divided by (model.hpp:20-26). */
CDFT_API int cdft_create_model(cdft_engine** out, const long shape[3], double dx, int n_species,
                               const double* diameters, int fmt_model, double esfmt_A, double esfmt_B,
                               int n_interactions, const cdft_model_interaction* interactions, double kT,
                               int precision, int batch);

/* Number of problems an engine evaluates per call. */
CDFT_API int cdft_engine_batch(const cdft_engine* engine, int* batch);

CDFT_API int cdft_destroy(cdft_engine* engine);

/* Engine facts: info = {N, Nk, S, n_channels, n_deriv_channels, precision,
 * kernels per evaluation, scratch bytes}. */
CDFT_API int cdft_engine_info(const cdft_engine* engine, long long info[8]);

/* a_vdw of interaction m as computed at set-up (InteractionWeight::a_vdw). */
CDFT_API int cdft_engine_a_vdw(const cdft_engine* engine, int m, double* a_vdw);

/* functionals::total (functionals.hpp:64-95) on HOST buffers:
 *   rho    : S*N doubles            vext : S*N doubles or NULL (zero field)
 *   mu     : S values (beta mu)     force: S*N doubles or NULL
 *   scalars: CDFT_SCALAR_COUNT doubles or NULL
 * Copies in, evaluates, copies out and synchronises. */
CDFT_API int cdft_total(cdft_engine* engine, const double* rho, const double* vext, const double* mu, double* force,
               double* scalars);

/* functionals::total for `count` states held in HOST memory, one after the
 * other, with the copies overlapped: the host->device copy of state i+1 and
 * the device->host copy of state i-1 run on their own streams while state i
 * is evaluated (two device slots alternate).  The same evaluation as count
 * cdft_total calls, the same results; returns when every result is in host
 * memory.  Page-locked host buffers let the copies overlap.
 *   rho    : count pointers to B*S*N doubles
 *   vext   : NULL (no field) or count pointers (entries may be NULL)
 *   mu     : count * B*S values (state i at mu + i*B*S)
 *   force  : NULL or count pointers (entries may be NULL: no force copy)
 *   scalars: NULL or count * B*CDFT_SCALAR_COUNT doubles
 * No reference counterpart: the reference evaluates one state per call
 * (functionals.hpp:64-95); this is that call for a stream of states. */
CDFT_API int cdft_total_stream(cdft_engine* engine, int count, const double* const* rho, const double* const* vext,
                               const double* mu, double* const* force, double* scalars);

/* functionals::total on DEVICE buffers, asynchronous on `stream`
 * (cudaStream_t; NULL = the legacy default stream).  rho, vext, force and
 * scalars are device pointers; mu is a host array read at call time. */
CDFT_API int cdft_total_device(cdft_engine* engine, const double* rho, const double* vext, const double* mu, double* force,
                      double* scalars, void* stream);


/* ---- drivers (device-resident; single species) --------------------------- */

/* FIRE2 parameters, fire.hpp:33-44 (same names and defaults). */
typedef struct {
  double dt, dt_max, dt_min, alpha_start, f_inc, f_dec, f_alpha;
  int n_delay, max_uphill;
  double force_tolerance;
  int max_steps;
} cdft_fire_params;

#define CDFT_MIN_GRAND_POTENTIAL 0
#define CDFT_MIN_FIXED_MASS 1
#define CDFT_MIN_SADDLE 2
#define CDFT_PARAM_UNBOUNDED 0
#define CDFT_PARAM_BOUNDED 1

/* Minimizer configuration (minimization.hpp:27-39, 123-147). */
typedef struct {
  cdft_fire_params fire;
  int mode;                 /* CDFT_MIN_* */
  int parametrization;      /* CDFT_PARAM_* */
  double rho_min, rho_max;  /* Unbounded{rho_min} / Bounded{rho_min, rho_max} */
  int homogeneous_boundary; /* Minimizer::use_homogeneous_boundary */
  double chemical_potential;
  double target_mass;       /* fixed mass / saddle */
  double boundary_mass;     /* saddle: mass of the boundary shell */
  int use_monitor;          /* 1: the minimiser's energy monitor; 0: rms force (Fire::step) */
  int check_interval;       /* device steps between host checks */
  /* external field of every evaluation: device, B * N doubles (the engine's
   * batch), or NULL.  The reference's Minimizer has none (init.hpp:28-58
   * drops V_ext); a hard wall or a trap needs it. */
  const double* external_field;
} cdft_minimizer_config;

typedef struct {
  double free_energy, grand_potential, rms_force;
  int iterations, converged, uphill_error;
} cdft_minimizer_result;

/* Minimizer::grand_potential / Minimizer::fixed_mass (minimization.hpp:182-354)
 * and the projected FIRE of Search::find (saddle_point.hpp:445-530, mode
 * CDFT_MIN_SADDLE with `direction`).  rho: N doubles on the device, replaced
 * by the minimiser's final density.  `refine` (or NULL): an FP64 engine of
 * the same model that takes over once the convergence measure (the monitor,
 * or the rms force when use_monitor is 0) drops below refine_switch *
 * force_tolerance, once it has not improved by 10% over 8 host checks (the
 * noise floor of mixed-precision forces), or once the run has converged
 * under the engine's own forces, and continues until the FP64 forces
 * converge too (mixed-precision defect correction).
 * Returns CDFT_ERR_RUNTIME with "fire::step: exceeded max uphill steps" where
 * the reference throws (fire.hpp:106-108). */
CDFT_API int cdft_minimize(cdft_engine* engine, const cdft_minimizer_config* cfg, double* rho,
                           const double* direction, cdft_engine* refine, double refine_switch,
                           cdft_minimizer_result* result, void* stream);

/* Minimizer::grand_potential / fixed_mass for every problem of a batched
 * engine (cdft_create_batch) at once.  rho: batch*N device doubles, replaced
 * by the results; mu: batch host values (beta mu); target_mass: batch host
 * values (fixed mass) or NULL; results: batch entries.  cfg->mode is
 * CDFT_MIN_GRAND_POTENTIAL or CDFT_MIN_FIXED_MASS; cfg->chemical_potential
 * and cfg->target_mass are not used.  Converged problems stop changing while
 * the others continue; an uphill error of one problem is reported in its
 * result (uphill_error = 1) without stopping the others.  `refine`: a
 * batched FP64 engine with the same batch, or NULL.  No reference
 * counterpart: the reference minimises one state per call. */
CDFT_API int cdft_minimize_batch(cdft_engine* engine, const cdft_minimizer_config* cfg, const double* mu,
                                 const double* target_mass, double* rho, cdft_engine* refine, double refine_switch,
                                 cdft_minimizer_result* results, void* stream);

/* One member of a group minimisation: the problems of one batched engine. */
typedef struct {
  cdft_engine* engine;          /* batch B (cdft_create_batch / cdft_create_model) */
  cdft_engine* refine;          /* FP64 engine of the same batch, or NULL */
  double refine_switch;
  const double* mu;             /* B host values (beta mu) */
  const double* target_mass;    /* B host values (fixed mass), or NULL */
  double* rho;                  /* B * N device doubles, replaced by the results */
  cdft_minimizer_result* results;  /* B entries */
} cdft_group_member;

/* Minimizer::grand_potential / fixed_mass for the problems of several
 * batched engines at once -- an uneven parameter sweep with one engine per
 * grid size (48^3, 64^3, 96^3 ...).  One FIRE step of every running member is
 * one launch of a CUDA graph whose branches run each member's step on its
 * own stream, so the grids share the GPU; every control decision is per
 * problem on the device and the host reads all control blocks every
 * cfg->check_interval steps.  A member leaves the graph when all its
 * problems have stopped.  cfg as cdft_minimize_batch (mode grand potential
 * or fixed mass; chemical_potential and target_mass unused).  Uphill errors
 * are reported per problem.  No reference counterpart: the reference
 * minimises one state per call (minimization.hpp:280-354). */
CDFT_API int cdft_minimize_group(int n_members, const cdft_group_member* members, const cdft_minimizer_config* cfg,
                                 void* stream);

/* DDFT step configuration, dynamics.hpp:26-33. */
typedef struct {
  double dt, diffusion_coefficient, min_density, dt_max, fp_tolerance;
  int fp_max_iterations;
} cdft_ddft_config;

/* integrating_factor_step (dynamics.hpp:333-401): one implicit step of rho
 * (device, N); cfg->dt is divided by 10 on every restart, as in the
 * reference.  energy: Omega after the step. */
CDFT_API int cdft_ddft_step(cdft_engine* engine, cdft_ddft_config* cfg, double chemical_potential, double* rho,
                            double* energy, int* fp_iterations, void* stream);

/* FP64 defect correction of the integrating-factor steps of a mixed-
 * precision engine (cdft_ddft_step, cdft_ddft_run, cdft_ddft_simulate): once
 * a step's fixed point has converged with `engine`, `iterations` (>= 0) more
 * fixed-point iterations run with the FP64 engine `refine` (same grid and
 * model, batch 1), which also gives the step's final forces and energy (with
 * 0 iterations only those).
 * refine NULL clears it.  No reference counterpart (the reference has one
 * precision). */
CDFT_API int cdft_ddft_set_refine(cdft_engine* engine, cdft_engine* refine, int iterations);

/* Facts of the engine's last integrating-factor step: info = {fixed-point
 * iterations, restarts, status (1 converged, 2 gave up after 64 restarts with
 * the last iterate), 1 if the fixed-point loop ran on the device as the
 * conditional WHILE node of the step's CUDA graph (0: host-driven)};
 * refine_deviation (or NULL): max |change| of the last FP64 refinement
 * iteration (0 without refinement). */
CDFT_API int cdft_ddft_last_step(cdft_engine* engine, int info[4], double* refine_deviation);

/* Simulation::run (dynamics.hpp:583-693) without snapshots: n_steps steps
 * with the adaptive dt (x2 after 5 successes, capped at dt_max).
 * times / energies: n_steps + 1 host doubles each, or NULL. */
CDFT_API int cdft_ddft_run(cdft_engine* engine, cdft_ddft_config* cfg, double chemical_potential, int n_steps,
                           double* rho, double* times, double* energies, void* stream);

/* split_operator_step (dynamics.hpp:410-465): Strang splitting, half a
 * diffusion step exp(-D k^2 dt / 2) in k-space, an explicit excess step,
 * half a diffusion step; every stage clamped at min_density.  rho (device, N)
 * is advanced in place; energy: Omega after the step.  cfg->dt is not
 * changed. */
CDFT_API int cdft_ddft_split_step(cdft_engine* engine, const cdft_ddft_config* cfg, double chemical_potential,
                                  double* rho, double* energy, void* stream);

/* crank_nicholson_step (dynamics.hpp:472-538): the fixed-point iteration
 * of the Crank-Nicolson update with continuous k^2; fp_iterations: the
 * iterations taken (or NULL). */
CDFT_API int cdft_ddft_cn_step(cdft_engine* engine, const cdft_ddft_config* cfg, double chemical_potential,
                               double* rho, double* energy, int* fp_iterations, void* stream);

/* Return non-zero from the stop callback to end a simulation after `step`. */
typedef int (*cdft_ddft_stop_fn)(int step, double time, double energy, void* user);

/* Simulation::run (dynamics.hpp:583-693) with snapshots: as cdft_ddft_run,
 * plus the density at step 0 and every snapshot_interval steps copied to
 * snapshots (host, snapshot_capacity * N doubles; pinned memory lets the
 * copies overlap the next steps) with their step numbers in snapshot_steps
 * (host, snapshot_capacity ints, or NULL); snapshots beyond the capacity
 * are dropped.  reservoir_mask (device, N bytes, or NULL): the cells that
 * reservoir_boundary (dynamics.hpp:551-557) resets to reservoir_density on
 * the initial state and after every step.  stop (or NULL) is called after
 * every step with the step, the time and Omega.  steps_done /
 * snapshot_count: the steps taken and the snapshots written. */
CDFT_API int cdft_ddft_simulate(cdft_engine* engine, cdft_ddft_config* cfg, double chemical_potential, int n_steps,
                                double* rho, double* times, double* energies, int snapshot_interval,
                                double* snapshots, int* snapshot_steps, int snapshot_capacity, int* snapshot_count,
                                const unsigned char* reservoir_mask, double reservoir_density,
                                cdft_ddft_stop_fn stop, void* user, int* steps_done, void* stream);

/* Picard parameters (picard.hpp:31-36; log_interval has no counterpart,
 * check_interval is how many iterations run between host checks of the
 * convergence flags; constraint_min_density is the min_density of
 * fixed_mass_constraint, minimization.hpp:159-164). */
typedef struct {
  double mixing, min_density, tolerance, constraint_min_density;
  int max_iterations, check_interval;
} cdft_picard_config;

typedef struct {
  double grand_potential, residual;
  int iterations, converged;
} cdft_picard_result;

/* Picard::solve (picard.hpp:63-124) for every problem of an engine (batch
 * B >= 1): rho <- max(rho exp(-mixing force / dV), min_density) until the
 * force RMS or the change of Omega falls below the tolerance.  mu: B host
 * values; target_mass: B host values, or NULL for no constraint; with it,
 * fixed_mass_constraint (minimization.hpp:159-180) rescales the excess over
 * background (device, B * N, or NULL for zero) after every update.  rho:
 * device, B * N.  results: B entries.  Converged problems stop changing
 * while the others continue. */
CDFT_API int cdft_picard(cdft_engine* engine, const cdft_picard_config* cfg, const double* mu,
                         const double* target_mass, const double* background, double* rho,
                         cdft_picard_result* results, void* stream);

/* Hessian-vector product hv = d(force)/d(rho) . v of Omega at rho (device
 * vectors, N each); `boundary` 1 zeroes the faces (the fixed boundary of
 * saddle_point.hpp:377-384).  Exact forward-over-reverse differentiation;
 * replaces hessian_times_vector (saddle_point.hpp:30-39). */
CDFT_API int cdft_hvp(cdft_engine* engine, const double* rho, const double* v, double chemical_potential,
                      int boundary, double* hv, void* stream);

/* The reference's finite-difference product (force(rho + eps v) - force_at_rho) / eps. */
CDFT_API int cdft_hvp_fd(cdft_engine* engine, const double* rho, const double* force_at_rho, const double* v,
                         double chemical_potential, double eps, int boundary, double* hv, void* stream);

/* EigenvalueSolver (saddle_point.hpp:158-276).  method
 * CDFT_EIGEN_RAYLEIGH_RITZ is the reference's 3-vector iteration;
 * CDFT_EIGEN_LANCZOS is block Lanczos on exact products (exact_hvp = 1) of
 * the fixed-boundary Hessian restricted to the interior (the same operator,
 * made symmetric): `block` directions per batched product (1..4), `max_basis`
 * blocks before a restart, the host reading the projected matrix every
 * `check_interval` products; zero fields take the defaults 1, 32 and 4. */
#define CDFT_EIGEN_RAYLEIGH_RITZ 0
#define CDFT_EIGEN_LANCZOS 1
typedef struct {
  double tolerance;
  int max_iterations;
  double hessian_eps;
  int exact_hvp;            /* 1: cdft_hvp, 0: finite differences as the reference */
  unsigned long long seed;  /* random initial vector */
  int method;               /* CDFT_EIGEN_* */
  int block, max_basis, check_interval;
} cdft_eigen_config;

/* Smallest eigenpair of the Hessian at rho (fixed boundary).  vec (device,
 * N): initial guess when use_guess, else drawn; receives the eigenvector. */
CDFT_API int cdft_eigen_solve(cdft_engine* engine, const cdft_eigen_config* cfg, const double* rho,
                              double chemical_potential, double* vec, int use_guess, double* eigenvalue,
                              int* iterations, int* converged, void* stream);

/* cdft_eigen_solve with a product engine for the Lanczos method: hvp_engine
 * (or NULL: `engine`, which then needs batch 1) is an engine of the same grid
 * and model whose batch equals cfg->block; its batched exact products at rho
 * drive the block recurrence (an FP64 product engine keeps the products in
 * FP64 under a mixed-precision `engine`).  Replaces EigenvalueSolver::solve
 * (saddle_point.hpp:171-276) with the same operator and outputs. */
CDFT_API int cdft_eigen_solve_ex(cdft_engine* engine, cdft_engine* hvp_engine, const cdft_eigen_config* cfg,
                                 const double* rho, double chemical_potential, double* vec, int use_guess,
                                 double* eigenvalue, int* iterations, int* converged, void* stream);

/* Search (saddle_point.hpp:324-353). */
typedef struct {
  cdft_fire_params fire;
  cdft_eigen_config eigen;
  double rho_min;
  double omega_tolerance, tolerance_start, tolerance_factor;
  int max_outer_iterations, eigenvalue_clear_count;
} cdft_saddle_config;

/* Search::find (saddle_point.hpp:367-589): eigenvector following at fixed
 * mass from rho (device, N, replaced by the saddle density); eigvec (device,
 * N) receives the unstable mode.  out = {grand_potential, eigenvalue}. */
CDFT_API int cdft_saddle_find(cdft_engine* engine, const cdft_saddle_config* cfg, double* rho,
                              double chemical_potential, double target_mass, double* eigvec, double out[2],
                              int* outer_iterations, int* converged, void* stream);

/* Search::find (saddle_point.hpp:367-589) with the mixed-precision and
 * batched-product options: `refine` (or NULL) is an FP64 engine that finishes
 * every projected FIRE run once its rms force is below refine_switch times
 * the run's tolerance (FP64 defect correction); `hvp_engine` (or NULL) the
 * product engine of a Lanczos eigen solve (cdft_eigen_solve_ex).
 * counts = {outer iterations, eigen products, FIRE steps} (or NULL). */
CDFT_API int cdft_saddle_find_ex(cdft_engine* engine, cdft_engine* refine, cdft_engine* hvp_engine,
                                 double refine_switch, const cdft_saddle_config* cfg, double* rho,
                                 double chemical_potential, double target_mass, double* eigvec, double out[2],
                                 int counts[3], int* converged, void* stream);

/* ---- bulk thermodynamics (host) ------------------------------------------ */

/* The uniform fluid of a functional: species diameters, FMT model and the
 * mean-field a_vdw of each interaction (BulkThermodynamics,
 * functionals/bulk/thermodynamics.hpp:201-206). */
typedef struct {
  int species_i;
  int species_j;
  double a_vdw;
} cdft_bulk_interaction;

typedef struct {
  int n_species;
  double diameters[CDFT_MAX_SPECIES];
  int fmt_model;
  double esfmt_A, esfmt_B;
  int n_interactions;
  cdft_bulk_interaction interactions[CDFT_MAX_INTERACTIONS];
} cdft_bulk_model;

/* Functional::bulk() (functional.hpp:48-50): the engine's model with the grid
 * a_vdw of its mean-field weights. */
CDFT_API int cdft_engine_bulk_model(const cdft_engine* engine, cdft_bulk_model* out);

/* f(rho) = ideal + hard-sphere + mean-field free energy density (kT units),
 * rho: n_species densities (thermodynamics.hpp:208-218). */
CDFT_API int cdft_bulk_free_energy_density(const cdft_bulk_model* model, const double* rho, double* f);

/* beta mu_s for every species (thermodynamics.hpp:220-244). */
CDFT_API int cdft_bulk_chemical_potentials(const cdft_bulk_model* model, const double* rho, double* mu);

/* beta P = sum rho_s mu_s - f (thermodynamics.hpp:246-253); Omega/V = -P. */
CDFT_API int cdft_bulk_pressure(const cdft_bulk_model* model, const double* rho, double* p);

/* density_from_chemical_potential (coexistence.hpp:35-49) for n targets at
 * once (one species): Newton from guess[i]; found[i] = 0 where the reference
 * returns nullopt (rho[i] is then NaN). */
CDFT_API int cdft_bulk_density_from_mu(const cdft_bulk_model* model, int n, const double* mu, const double* guess,
                                       int max_iterations, double tolerance, double* rho, int* found);

/* PhaseSearch::find_spinodal (coexistence.hpp:77-113): out = {rho_low,
 * rho_high}; found = 0 where the reference returns nullopt. */
CDFT_API int cdft_bulk_spinodal(const cdft_bulk_model* model, double rho_max, double rho_scan_step, double out[2],
                                int* found);

/* PhaseSearch::find_coexistence (coexistence.hpp:115-191): out = {rho_vapor,
 * rho_liquid}; max_iterations / tolerance are the Newton settings of the
 * PhaseSearch (the reference's defaults: 200, 1e-10). */
CDFT_API int cdft_bulk_coexistence(const cdft_bulk_model* model, double rho_max, double rho_scan_step,
                                   int max_iterations, double tolerance, double out[2], int* found);

/* ---- allocation-free entry point ------------------------------------------ */

/* The ideal-gas and external-field terms (ideal_gas.hpp:18-37 and
 * external_field.hpp:16-30) for callers that cannot allocate device memory:
 * no engine, no cudaMalloc, no cuFFT.  No counterpart in the reference; it is
 * the local-term part of the pointwise kernel behind cdft_total.
 *   rho, vext (or NULL), force: n_species * n_points device doubles
 *   mu: n_species host values (beta mu);  scalars: 2 + n_species device
 *   doubles receiving [F_id, F_ext, N_0 .. N_{S-1}] (the entries 2, 3 and
 *   6.. of cdft_total's scalar block).
 * force = (ln max(rho, 1e-300) - mu + V) dV.  Scratch is a 28 KiB file-scope
 * device array (592 x 6 partial sums) held by every GPU that loads the
 * library; n_species is limited to 4 by it.  Every call looks the array's
 * address up (cudaGetSymbolAddress, so a device reset is harmless); the first
 * call on a device also loads the module there: make that first call before
 * any stream capture.  All calls share the array: calls whose kernels overlap
 * on the GPU race, so serialise them.  Asynchronous on `stream`. */
CDFT_API int cdft_local_terms_noalloc(const double* rho, const double* vext, const double* mu, int n_species,
                                      long long n_points, double dv, double* force, double* scalars, void* stream);

/* Stage timing (a measurement hook; no reference counterpart).  With `on`,
 * every evaluation records CUDA events between its stages on its own stream
 * (a ring of 64 event sets: evaluations still queue back to back; the host
 * waits only when the ring is full); off by default.  The stages, in order:
 * 0 split / FP32 conversion (mixed), 1 r2c rho, 2 k_forward, 3 c2r channels,
 * 4 pointwise, 5 r2c derivatives, 6 k_backward, 7 c2r force, 8 epilogue
 * (which also finishes the scalars), 9 reserved (empty). */
#define CDFT_STAGE_COUNT 10
CDFT_API int cdft_engine_stage_timing(cdft_engine* engine, int on);

/* Accumulated milliseconds per stage since the last call, and the number of
 * timed evaluations; clears the accumulators. */
CDFT_API int cdft_engine_stage_times(cdft_engine* engine, double ms[CDFT_STAGE_COUNT], long long* evaluations);

/* Transform implementation of an engine (no reference counterpart; the
 * reference uses FFTW).  CDFT_TRANSFORMS_FUSED: hand-written plane / column
 * FFT kernels with the k-space stages fused into the column pass, available
 * for mixed-precision engines whose nx, ny and nz are each one of 16, 32,
 * 48, 64, 96 or 128 (and whose channel tiles fit in shared memory), and the
 * default there.
 * CDFT_TRANSFORMS_CUFFT: cuFFT plans with separate k-space kernels (every
 * other engine, and the exact HVP always).  Selecting FUSED where it is not
 * available is CDFT_ERR_INVALID. */
#define CDFT_TRANSFORMS_CUFFT 0
#define CDFT_TRANSFORMS_FUSED 1
CDFT_API int cdft_engine_set_transforms(cdft_engine* engine, int transforms);

/* The current transform implementation and whether FUSED is available. */
CDFT_API int cdft_engine_transforms(const cdft_engine* engine, int* transforms, int* fused_available);

/* Plane chunks of the fused path (no reference counterpart; execution
 * tuning only, results unchanged but for the summation order of the
 * scalars).  The inverse plane pass, the pointwise stage and the derivative
 * plane pass run as `chunks` groups of nx / chunks x planes on
 * engine-owned streams forked from the caller's stream, so one group's FP64
 * pointwise work overlaps another's FP32 transforms; 1 runs them back to
 * back.  chunks in 1..CDFT_MAX_PLANE_CHUNKS dividing nx; the default is 4
 * from nx = 64 on, else 1.  CDFT_ERR_INVALID on an engine without the fused
 * path or for another count. */
#define CDFT_MAX_PLANE_CHUNKS 8
CDFT_API int cdft_engine_set_plane_chunks(cdft_engine* engine, int chunks);

/* Autotuner (no reference counterpart): times every plane-chunk count (1, 2,
 * 4, 8 dividing nx) of the fused path on the caller's device state (rho and
 * vext as for cdft_total_device, vext may be NULL; mu: B*S host values or
 * NULL for zeros), `reps` evaluations each after two untimed ones, and keeps
 * the fastest for this engine and for every engine created later in this
 * process with the same grid, species count, batch, model and interaction
 * count.  chunks (out, optional): the count chosen.  ms (out, optional,
 * CDFT_MAX_PLANE_CHUNKS entries): ms[k - 1] is the time per evaluation of
 * count k, 0 where not tried.  Synchronises the stream; the engine's scratch
 * force and scalars are overwritten.  An engine without the fused path
 * returns CDFT_OK, its current count and no timings. */
CDFT_API int cdft_engine_autotune(cdft_engine* engine, const double* rho, const double* vext, const double* mu,
                                  void* stream, int reps, int* chunks, double* ms);

/* The pointwise kernel of the TMA-staged path (no reference counterpart):
 * 0 the generic kernel; 1 .. 5 the kernel specialised for one species and
 * at most two interactions (mixed precision): 1 and 2 with its registers
 * sized for 5 or 6 CTAs per SM; 3 (5 CTAs per SM), 4 and 5 (two points per
 * thread, 3 or 4 CTAs per SM) take a branch-free FP64 path in warps whose
 * points all have eta >= 1e-6 (one reciprocal for 1/eta and 1/(1 - eta)).
 * Every variant gives the same results up to the rounding of the pointwise
 * FP64 arithmetic.  available (out): 1 where 1 .. 5 exist.  The column passes of an engine with several species run tiles of
 * 16 or (where the spectra fit in shared memory) 32 in-plane columns; one
 * species always 16 (cdft_engine_set_column_tile / cdft_engine_column_tile;
 * 0 without the fused path).  Each plane chunk's pointwise launch takes the
 * full pointwise grid divided by d = min(spread, chunks); spread 0 (the
 * default) divides it by the chunk count, 1, 2, 4, 8 give a chunk a larger
 * share (cdft_engine_set_pointwise_spread / cdft_engine_pointwise_spread).
 * cdft_engine_autotune times every pointwise variant, column tile width and
 * spread with every plane-chunk count and keeps the fastest combination;
 * cdft_engine_autotune_ex also returns the whole table:
 * ms[((t * CDFT_POINTWISE_VARIANTS + v) * CDFT_MAX_PLANE_CHUNKS + k - 1)
 *    * CDFT_POINTWISE_SPREADS + log2 d]
 * for tile index t (0: 16, 1: 32), variant v, k chunks and spread d (0
 * where not tried; 2 * CDFT_POINTWISE_VARIANTS * CDFT_MAX_PLANE_CHUNKS *
 * CDFT_POINTWISE_SPREADS entries), choice = {chunks, variant, tile, spread};
 * the middle plane width kept is read with cdft_engine_plane_width. */
#define CDFT_POINTWISE_VARIANTS 6
#define CDFT_POINTWISE_SPREADS 4
CDFT_API int cdft_engine_set_pointwise(cdft_engine* engine, int variant);
CDFT_API int cdft_engine_pointwise(const cdft_engine* engine, int* variant, int* available);
CDFT_API int cdft_engine_set_column_tile(cdft_engine* engine, int tile);
CDFT_API int cdft_engine_column_tile(const cdft_engine* engine, int* tile);
/* Threads per plane CTA of the fused path's two middle plane passes (the
 * inverse transforms of the weighted-density channels and the forward
 * transforms of the derivative channels, one CTA per x plane and channel):
 * wide = 0 the base width (512 threads at 128 x 128 planes), 1 twice that.
 * Results are bitwise the same.  cdft_engine_autotune times both; its table
 * holds the faster one per entry.  cdft_engine_plane_width gives -1 without
 * the fused path. */
CDFT_API int cdft_engine_set_plane_width(cdft_engine* engine, int wide);
CDFT_API int cdft_engine_plane_width(const cdft_engine* engine, int* wide);
CDFT_API int cdft_engine_set_pointwise_spread(cdft_engine* engine, int spread);

/* Programmatic dependent launch between consecutive passes of the fused path
 * (a pass may be scheduled while its predecessor in the stream finishes and
 * waits in the kernel for its completion): on = 1 (default) or 0, -1 leaves
 * it; was (optional) receives the setting before the call.  Results are
 * the same either way; it is off while stage timing runs (captured graphs
 * keep the launches as programmatic edges). */
CDFT_API int cdft_engine_set_dependent_launch(cdft_engine* engine, int on, int* was);

/* Anchored split (no reference counterpart; mixed-precision engines): the
 * mixed path transforms rho - mean in FP32, so its round-off scales with the
 * density's own swing, which for a solid is the peak height.  From
 * cdft_engine_set_anchor on, an evaluation instead transforms rho - rho_a in
 * FP32 and adds, point by point, the FP64 weighted densities, derivative
 * channels and back-convolution of the anchor state rho_a, evaluated once
 * here by fp64_engine (an FP64 engine of the same grid, species, model,
 * interactions and batch): near the anchor the error scales with
 * |rho - rho_a|.  rho_anchor: device, B*S*N doubles (copied).  Anchored
 * evaluations run the cuFFT transforms and the generic pointwise kernel;
 * the HVP keeps the mean split.  Synchronises `stream`.
 * cdft_engine_clear_anchor returns to the mean split. */
CDFT_API int cdft_engine_set_anchor(cdft_engine* engine, cdft_engine* fp64_engine, const double* rho_anchor,
                                    void* stream);
/* The same with rho_anchor in HOST memory (B*S*N doubles). */
CDFT_API int cdft_engine_set_anchor_host(cdft_engine* engine, cdft_engine* fp64_engine, const double* rho_anchor);
CDFT_API int cdft_engine_clear_anchor(cdft_engine* engine);
CDFT_API int cdft_engine_anchored(const cdft_engine* engine, int* anchored);
CDFT_API int cdft_engine_pointwise_spread(const cdft_engine* engine, int* spread);
CDFT_API int cdft_engine_autotune_ex(cdft_engine* engine, const double* rho, const double* vext, const double* mu,
                                     void* stream, int reps, int choice[4], double* ms);

/* Step graphs (no reference counterpart; execution mode, process-wide): the
 * FIRE minimisers (cdft_minimize, cdft_minimize_batch, the saddle search's
 * FIRE) capture one step (the FIRE update and the evaluation) as a CUDA graph
 * and replay it every step, and the DDFT integrating-factor step
 * (cdft_ddft_step, cdft_ddft_simulate) each fixed-point iteration, on a
 * driver-owned stream joined to the caller's stream by events.  On by default; results are identical either way.  Off
 * while an engine records stage timings. */
CDFT_API int cdft_set_step_graphs(int on);
CDFT_API int cdft_step_graphs(int* on);

/* Status of earlier asynchronous calls on `stream`: CDFT_ERR_RUNTIME if a
 * bounded device-side wait gave up (the scalars of that call are NaN), else
 * CDFT_OK.  Synchronises the stream and clears the flag.  No reference
 * counterpart: the reference is synchronous CPU code. */
CDFT_API int cdft_engine_status(cdft_engine* engine, void* stream);

/* ------------------------------------------------------------ lattices */

/* Structure, Orientation and ExportFormat (types.hpp:52-71). */
#define CDFT_BCC 0
#define CDFT_FCC 1
#define CDFT_HCP 2
#define CDFT_ORIENT_001 0
#define CDFT_ORIENT_010 1
#define CDFT_ORIENT_100 2
#define CDFT_ORIENT_110 3
#define CDFT_ORIENT_101 4
#define CDFT_ORIENT_011 5
#define CDFT_ORIENT_111 6
#define CDFT_EXPORT_XYZ 0
#define CDFT_EXPORT_CSV 1

/* The number of sites build_lattice makes: sites per unit cell x
 * shape[0] x shape[1] x shape[2] (shape: 3 cell counts). */
CDFT_API int cdft_lattice_size(int structure, int orientation, const long* shape, long* n_sites);

/* build_lattice (crystal.cpp:205-245): site positions (host, row-major
 * n_sites x 3, `capacity` >= n_sites) with unit nearest-neighbour distance,
 * cells tiled x-fastest; dimensions (3 doubles, or NULL): the box edges.
 * Invalid shapes and HCP along 110/101/011/111 are CDFT_ERR_INVALID, as the
 * reference's std::invalid_argument. */
CDFT_API int cdft_build_lattice(int structure, int orientation, const long* shape, double* positions, long capacity,
                                double* dimensions);

/* Lattice::export_to (crystal.cpp:257-279): XYZ ("Ar x y z" lines after the
 * count and a comment line) or CSV (header "x,y,z"), default stream
 * formatting.  A file that cannot be opened is CDFT_ERR_RUNTIME. */
CDFT_API int cdft_lattice_export(const double* positions, long n_sites, const char* filename, int format);

/* A crystal density profile on the grid (device, N doubles, z-fastest):
 * rho = background + amplitude * sum_i exp(-alpha |r - R_i|^2) over the
 * sites (host, n_sites x 3) at minimum-image distance, each peak cut where
 * alpha |r - R_i|^2 > 40.  The box must be at least 2 sqrt(40 / alpha) on
 * every axis.  No reference counterpart (a project-defined initialiser of
 * solid profiles from build_lattice sites). */
CDFT_API int cdft_gaussian_peaks(const long* shape, double dx, const double* sites, long n_sites, double alpha,
                                 double amplitude, double background, double* rho, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CDFT_B200_H */
