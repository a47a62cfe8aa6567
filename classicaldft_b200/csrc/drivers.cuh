// Device-resident drivers of the functional: FIRE2 minimisation (grand
// potential, fixed mass, projected saddle mode), DDFT integrating-factor
// steps, Hessian-vector products and the smallest-eigenpair solver.
//
// Every vector lives in HBM; per-step control decisions (the FIRE2 power test,
// dt / alpha updates, convergence monitor) are taken by single-thread device
// kernels from reduced scalars, so a FIRE step is a fixed kernel sequence that
// never waits on the host.  The host reads the small control block only every
// `check_interval` steps.
#pragma once

#include <cufft.h>

#include <memory>
#include <vector>

#include "cdft_common.cuh"
#include "engine.cuh"

namespace cdft {

// fire.hpp:33-44 (parameters)
struct FireParams {
  double dt = 1e-3, dt_max = 1e-2, dt_min = 1e-8;
  double alpha_start = 0.1, f_inc = 1.1, f_dec = 0.5, f_alpha = 0.99;
  int n_delay = 5, max_uphill = 20;
  double force_tolerance = 0.1;
  int max_steps = 10000;
};

enum FireMode : int { kGrandPotential = 0, kFixedMass = 1, kSaddle = 2 };
enum ParamKind : int { kUnbounded = 0, kBounded = 1 };

// Device-side FIRE2 state of one problem (fire.hpp:15-26 plus the
// minimiser's monitor); a batched engine keeps one per problem.
struct FireDevState {
  double dt, alpha;
  int n_positive, n_negative, iteration, converged;
  int active;      // 1 while steps still change the state
  int backtrack;   // this step backtracks (power <= 0)
  int uphill_error;
  double dt_prev;  // dt before this step's update (the backtrack uses it)
  double energy, rms_force, vv, monitor;
  double ratio;    // |v| / |f| of the mixing step
  double scale;    // density rescale of the fixed-mass / saddle compute
  double lambda;   // Lagrange multiplier of the fixed-mass / saddle compute
  double free_energy;
  double target_mass;  // fixed mass / saddle target of this problem
  double bavg;         // mean boundary force of the last compute
  double f2;           // |f|^2 of the forces driving this step
};

struct FireConfig {
  FireParams fire;
  int mode = kGrandPotential;
  int param = kUnbounded;
  double rho_min = 1e-18, rho_max = 1.0;
  bool homogeneous_boundary = true;
  double mu = 0.0;
  double target_mass = 0.0;     // fixed mass
  double boundary_mass = 0.0;   // saddle: mass held by the boundary shell
  int check_interval = 25;
  bool use_monitor = true;      // Minimizer convergence (minimization.hpp:431-434) vs rms (fire.hpp:162)
  // External field of every evaluation (device, B*N, or null).  The
  // reference's Minimizer evaluates without one (init::from_profile drops
  // V_ext, init.hpp:28-58); a wall or a trap needs it.
  const double* vext = nullptr;
};

struct FireResult {
  double free_energy = 0.0, grand_potential = 0.0, rms_force = 0.0;
  int iterations = 0;
  bool converged = false;
  bool uphill_error = false;
};

class Drivers;

// One member of a group minimisation: the problems of one batched engine
// (grand potential or fixed mass, as fire_minimize_batch).
struct GroupMember {
  Drivers* drivers = nullptr;
  const double* mu = nullptr;    // B host values
  const double* mass = nullptr;  // B host values (fixed mass) or null
  double* rho = nullptr;         // B*N device doubles, replaced by the results
  Engine* refine = nullptr;      // FP64 engine of the same batch, or null
  double refine_switch = 10.0;
};

// Minimisations of several batched engines -- typically one per grid size of
// an uneven parameter sweep -- advanced together: one step of every running
// member is ONE launch (a CUDA graph whose branches run each member's step
// on its own stream, so small grids fill the SMs beside large ones), the
// host checks every member's control blocks every check_interval steps, and
// a member leaves the graph when all its problems have stopped (the graph is
// captured again then, and when a member switches to its FP64 engine).
// Returns each member's results in member order.
std::vector<std::vector<FireResult>> fire_minimize_group(std::vector<GroupMember>& members, const FireConfig& cfg,
                                                         cudaStream_t stream);

// Process-wide switch: the minimisers replay each step as a captured CUDA
// graph (default on; results are the same either way).
void set_step_graphs(bool on);
bool step_graphs();

struct FireRun;

class Drivers {
 public:
  explicit Drivers(Engine& engine);
  ~Drivers();
  Drivers(const Drivers&) = delete;
  Drivers& operator=(const Drivers&) = delete;

  // Minimizer::grand_potential / fixed_mass (minimization.hpp:182-354) and the
  // saddle FIRE of Search::find (saddle_point.hpp:445-530).  rho: N doubles on
  // the device, replaced by the result.  `direction` (saddle mode, N doubles,
  // device) is the unit eigen-direction in parameter space, or null.
  // `refine` (optional) is an FP64 engine that takes over for the last
  // `refine_steps` steps after the monitor first drops below
  // `refine_switch` times the tolerance (mixed-precision defect correction).
  FireResult fire_minimize(const FireConfig& cfg, double* rho, const double* direction, cudaStream_t stream,
                           Engine* refine = nullptr, double refine_switch = 10.0);

  // The same minimisation for every problem of a batched engine at once
  // (grand potential or fixed mass; no saddle mode): problem b has chemical
  // potential mu[b] and (fixed mass) target mass[b], host arrays of B values;
  // rho holds B*N device doubles.  The FP64 `refine` engine (same batch)
  // takes over once every active problem's monitor is below refine_switch
  // times the tolerance.  Problems that converge stop changing while the
  // others continue.  Uphill errors are reported per problem.
  std::vector<FireResult> fire_minimize_batch(const FireConfig& cfg, const double* mu, const double* mass,
                                              double* rho, cudaStream_t stream, Engine* refine = nullptr,
                                              double refine_switch = 10.0);

  // DDFT integrating-factor step (dynamics.hpp:333-401) for one species;
  // returns the energy after the step and updates dt in place (dt/10 on
  // restart).  rho: N doubles, device.
  struct DDFTConfig {
    double dt = 1e-4, diffusion = 1.0, min_density = 1e-18, dt_max = 1.0, fp_tolerance = 1e-4;
    int fp_max_iterations = 100;
    double mu = 0.0;
  };
  // The whole step runs on the device: with step graphs on (the default) it
  // is one CUDA graph whose fixed-point loop is a conditional WHILE node, the
  // restart decisions (negative density, growing deviation, no convergence
  // in fp_max_iterations: dt /= 10 and start again) taken by a one-thread
  // control kernel that also ends the loop; after kMaxRestarts restarts the
  // step gives up with the last iterate, as the host loop did.  With graphs
  // off the host launches the same kernels iteration by iteration.
  static constexpr int kMaxRestarts = 64;
  double ddft_step(DDFTConfig& cfg, double* rho, cudaStream_t stream, int* fp_iterations = nullptr);
  // FP64 defect correction of a mixed-precision IF step: after the fixed
  // point has converged with this driver's engine, `iterations` (>= 0) more
  // iterations use the FP64 `refine` engine (same model), which also gives
  // the step's final forces and energy (0: only that).  Null clears it.
  // Applies to ddft_step and ddft_run.
  void set_ddft_refine(Engine* refine, int iterations);
  // Facts of the last IF step: fixed-point iterations, restarts, status
  // (1 converged, 2 gave up after kMaxRestarts), 1 if the loop ran as a
  // device-side conditional node, and the deviation of the last FP64
  // refinement iteration (0 without one).
  struct DDFTStepInfo {
    int fp_iterations = 0, restarts = 0, status = 0, device_loop = 0;
    double refine_deviation = 0.0;
  };
  const DDFTStepInfo& last_ddft_step() const { return ddft_info_; }

  // split_operator_step (dynamics.hpp:410-465): half diffusion in k-space,
  // forward-Euler excess step, half diffusion; returns the energy after it.
  double ddft_split_step(const DDFTConfig& cfg, double* rho, cudaStream_t stream);
  // crank_nicholson_step (dynamics.hpp:472-538), fixed-point iterated.
  double ddft_cn_step(const DDFTConfig& cfg, double* rho, cudaStream_t stream, int* fp_iterations = nullptr);

  // Simulation::run (dynamics.hpp:583-693) on the device: n_steps IF steps
  // with the adaptive dt; times / energies (n_steps + 1 host doubles each, or
  // null) get every step; every snapshot_interval steps (and at step 0) the
  // density is copied to the snapshot sink (host memory; the copy overlaps
  // the next step when that memory is page-locked); `stop` (or null) ends
  // the run after the step for which it returns nonzero.  Returns the steps
  // taken.
  struct SnapshotSink {
    double* host = nullptr;  // capacity * N doubles
    int* steps = nullptr;    // capacity step numbers
    int capacity = 0;
    int count = 0;           // written by ddft_run
  };
  using StopFn = int (*)(int step, double time, double energy, void* user);
  // reservoir_boundary (dynamics.hpp:551-557): cells with mask[i] != 0
  // (device, N bytes) reset to `density` on the initial state and after
  // every step.
  struct Reservoir {
    const unsigned char* mask = nullptr;
    double density = 0.0;
  };
  // Returns the steps taken (n_steps unless stop ended the run).
  int ddft_run(DDFTConfig& cfg, int n_steps, double* rho, double* times, double* energies, int snapshot_interval,
               SnapshotSink* snaps, StopFn stop, void* user, const Reservoir* reservoir, cudaStream_t stream);

  // Picard::solve (picard.hpp:63-124) for every problem of the engine's
  // batch: rho *= exp(-mixing force / dV), clamped at min_density, until the
  // rms force or the change of Omega is below the tolerance; with `mass`
  // (B values, or null) the fixed-mass constraint of
  // minimization.hpp:159-180 (relative to `background`, B*N device doubles,
  // or zero) after every update.
  struct PicardConfig {
    double mixing = 0.01, min_density = 1e-30, tolerance = 1e-6, constraint_min_density = 1e-30;
    int max_iterations = 5000, check_interval = 25;
  };
  struct PicardResult {
    double grand_potential = 0.0, residual = 0.0;
    int iterations = 0;
    bool converged = false;
  };
  std::vector<PicardResult> picard(const PicardConfig& cfg, const double* mu, const double* mass,
                                   const double* background, double* rho, cudaStream_t stream);

  // H v at rho (single species): exact forward-over-reverse (hvp_exact) or the
  // reference's finite difference (F(rho + eps v) - F(rho)) / eps.
  // `boundary` 1: fixed boundary (forces zeroed on the faces, saddle_point.hpp:382).
  void hvp_fd(const double* rho, const double* force_at_rho, const double* v, double* hv, double eps, double mu,
              int boundary, cudaStream_t stream);
  void hvp_exact(const double* rho, const double* v, double* hv, double mu, int boundary, cudaStream_t stream);

  // Plain force of one species with the boundary treatment (0 none, 1 fixed).
  double force(const double* rho, double* f, double mu, int boundary, cudaStream_t stream);

  // Device vector helpers (dot products etc.) used by the eigen solvers.
  double dot(const double* a, const double* b, long long n, cudaStream_t stream);
  void axpby(double a, const double* x, double b, double* y, long long n, cudaStream_t stream);  // y = a x + b y

  // EigenvalueSolver::solve (saddle_point.hpp:171-276): smallest eigenpair of
  // the Hessian of Omega at rho (fixed boundary on the forces), by the
  // reference's 3-vector Rayleigh-Ritz iteration.  `vec` (device, N) holds
  // the initial guess if `use_guess`, else a seeded normal vector is drawn;
  // it receives the unit eigenvector.
  // method kRayleighRitz is the reference's solver; kLanczos the block
  // Lanczos of lanczos.cuh on exact products (block directions per batched
  // product; the product engine's batch must equal `block`).
  enum EigenMethod : int { kRayleighRitz = 0, kLanczos = 1 };
  struct EigenConfig {
    double tolerance = 1e-4;
    int max_iterations = 300;
    double hessian_eps = 1e-6;
    int exact_hvp = 0;
    unsigned long long seed = 42;
    int method = kRayleighRitz;
    int block = 1;
    int max_basis = 32;
    int check_interval = 4;
  };
  struct EigenResult {
    double eigenvalue = 0.0;
    int iterations = 0;
    bool converged = false;
  };
  // `hvp_engine` (Lanczos only; null: this driver's engine, batch 1): an
  // engine of the same model whose batch is the Lanczos block size, used for
  // the batched exact products (an FP64 engine gives FP64 products under a
  // mixed-precision driver).
  EigenResult eigen_solve(const EigenConfig& cfg, const double* rho, double mu, double* vec, bool use_guess,
                          cudaStream_t stream, Engine* hvp_engine = nullptr);

  // Search::find (saddle_point.hpp:324-589): eigenvector following at fixed
  // mass.  rho (device, N) is replaced by the saddle density, eigvec (device,
  // N) receives the unstable direction.
  struct SaddleConfig {
    FireParams fire;
    EigenConfig eigen;
    double rho_min = 1e-18;
    double omega_tolerance = 1e-5, tolerance_start = 1e-3, tolerance_factor = 10.0;
    int max_outer_iterations = 20, eigenvalue_clear_count = 2;
  };
  struct SaddleResult {
    double grand_potential = 0.0, eigenvalue = 0.0;
    int outer_iterations = 0;
    bool converged = false;
    int eigen_iterations = 0;  // summed over the outer iterations
    int fire_steps = 0;        // summed over the outer iterations
  };
  // `refine`: an FP64 engine that finishes each projected FIRE run (mixed-
  // precision defect correction, as fire_minimize); `hvp_engine`: the
  // product engine of a Lanczos eigen solve (see eigen_solve).
  SaddleResult saddle_find(const SaddleConfig& cfg, double* rho, double mu, double target_mass, double* eigvec,
                           cudaStream_t stream, Engine* refine = nullptr, Engine* hvp_engine = nullptr,
                           double refine_switch = 10.0);

  Engine& engine() { return eng_; }

  // The FIRE loop in pieces, for driving several drivers together (a group
  // minimisation whose steps are one graph over every member):
  //   fire_begin      initial compute (fire.hpp:60-84) of a run
  //   fire_launch_step one step of every problem with the engine now evaluating
  //   fire_read_state  async D2H of the control blocks (the caller syncs)
  //   fire_decide      the host's check after that sync: the FP64 switch of
  //                    the refine engine (engine_changed), and the steps to
  //                    launch before the next check (0: the run is over)
  //   fire_advance     count launched steps
  //   fire_finish      final compute and results (synchronises the stream)
  void fire_begin(const FireConfig& cfg, const double* mu, const double* mass, double* rho, const double* direction,
                  cudaStream_t stream, Engine* refine, double refine_switch);
  void fire_launch_step(cudaStream_t stream);
  void fire_read_state(cudaStream_t stream);
  int fire_decide(cudaStream_t stream, bool* engine_changed);
  void fire_advance(int steps);
  const Engine* fire_engine() const;
  std::vector<FireResult> fire_finish(cudaStream_t stream);
  int batch() const { return B_; }
  // this driver's own stream for graph capture (created on first use)
  cudaStream_t graph_stream() {
    ensure_graph_stream();
    return graph_stream_;
  }

 private:
  void fire_compute(int initial, cudaStream_t stream);
  void capture_step(cudaStream_t stream);
  std::unique_ptr<FireRun> run_;
  std::vector<FireResult> fire_run(const FireConfig& cfg, const double* mu, const double* mass, double* rho,
                                   const double* direction, cudaStream_t stream, Engine* refine,
                                   double refine_switch);
  std::vector<FireResult> fire_loop(const FireConfig& cfg, const double* mu, const double* mass, double* rho,
                                    const double* direction, cudaStream_t stream, Engine* refine,
                                    double refine_switch, bool graphs);
  // CUDA graph of one FIRE step (captured on graph_stream_, replayed per
  // step; recaptured when the evaluating engine changes)
  cudaStream_t graph_stream_ = nullptr;
  cudaEvent_t graph_ev_[2] = {};
  cudaGraph_t step_graph_ = nullptr;
  cudaGraphExec_t step_exec_ = nullptr;
  const void* step_key_ = nullptr;
  void reset_step_graph();
  void ensure_graph_stream();
  // CUDA graph of one IF step, its device-side control state and its key
  // (everything baked into its kernel arguments)
  cudaGraph_t fp_graph_ = nullptr;
  cudaGraphExec_t fp_exec_ = nullptr;
  struct DDFTGraphKey {
    double mu = 0.0, tol = 0.0, min_density = 0.0, diffusion = 0.0;
    int fp_max = 0, refine_iterations = 0;
    const Engine* refine = nullptr;
    unsigned long long gen = 0, refine_gen = 0;
    bool operator==(const DDFTGraphKey& o) const {
      return mu == o.mu && tol == o.tol && min_density == o.min_density && diffusion == o.diffusion &&
             fp_max == o.fp_max && refine_iterations == o.refine_iterations && refine == o.refine && gen == o.gen &&
             refine_gen == o.refine_gen;
    }
  } fp_key_;
  void reset_fp_graph();
  void ddft_prologue(const DDFTConfig& cfg, cudaStream_t s);
  void ddft_body(const DDFTConfig& cfg, cudaStream_t s, unsigned long long cond, int use_cond);
  void ddft_epilogue(const DDFTConfig& cfg, cudaStream_t s);
  void capture_ddft_step(const DDFTConfig& cfg);
  void* ddft_st_ = nullptr;       // device control state of the IF step
  void* ddft_st_host_ = nullptr;  // pinned copy
  Engine* ddft_refine_ = nullptr;
  int ddft_refine_iterations_ = 0;
  DDFTStepInfo ddft_info_;

  Engine& eng_;
  long long N_ = 0;
  int B_ = 1;                 // problems of the engine's batch
  double* x_ = nullptr;       // FIRE parameters (B*N)
  double* v_ = nullptr;       // FIRE velocity (B*N)
  double* f_ = nullptr;       // FIRE force (parameter space, B*N)
  double* grad_ = nullptr;    // functional force from the engine (B*N)
  double* tmp_ = nullptr;     // scratch vector (HVP, DDFT)
  double* tmp2_ = nullptr;
  double* scalars_ = nullptr; // engine scalar blocks (B)
  double* red_ = nullptr;     // reduction partials [B][grid_][4]
  double* red_out_ = nullptr; // reduced values [B][8]
  FireDevState* st_ = nullptr;       // [B]
  FireDevState* st_host_ = nullptr;  // pinned [B]
  double* host_pin_ = nullptr;       // pinned scalars
  int grid_ = 0;              // CTAs per problem of the vector kernels
  // DDFT
  void* ddft_k_ = nullptr;    // 3 * Nk complex (rho0_k, R0_k, R1_k / work)
  double* lam_ = nullptr;     // nx + ny + nzh Laplacian eigenvalues
  cufftHandle plan_r2c_ = 0, plan_c2r_ = 0;
  cudaStream_t copy_stream_ = nullptr;          // snapshot D2H copies
  double* snap_stage_[2] = {nullptr, nullptr};  // device staging of two snapshots in flight
  cudaEvent_t snap_ready_[2] = {}, snap_done_[2] = {};
  void* fft_work_ = nullptr;
  bool ddft_ready_ = false;
  void ensure_ddft();
  // eigen solver vectors
  double* ev_[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  void* tan_ = nullptr;
};

}  // namespace cdft
