// The evaluation engine: one grid, its species, FMT model and mean-field
// interactions, with every buffer, cuFFT plan and weight resident in HBM.
//
// An Engine is what the reference's (Model, Weights) pair becomes on the GPU
// (include/dft/functionals/functionals.hpp:19-33): built once, immutable
// afterwards, evaluated many times.  It is not thread-safe: one stream per
// engine, as FFTW plans are per-object in the reference.
#pragma once

#include <cufft.h>

#include <string>
#include <vector>

#include "cdft_common.cuh"
#include "fft_core.cuh"
#include "fused.cuh"
#include "physics.hpp"

namespace cdft {

enum Precision : int { kFP64 = 0, kMixed = 1 };

struct PointwiseArgs;

struct InteractionSpec {
  int species_i = 0, species_j = 0;
  std::vector<double> weight_real;  // N doubles: cell weight * dV / N (mean_field.hpp:188)
  double a_vdw = 0.0;
  // on_device: weight_real and a_vdw are left empty and the engine builds
  // them from the potential, split and weight scheme at temperature kT
  bool on_device = false;
  Potential potential;
  int split = kWeeksChandlerAndersen, scheme = kWeightQuadraticF;
  double kT = 1.0;
};

struct EngineSpec {
  long shape[3] = {0, 0, 0};
  double dx = 0.0;
  std::vector<double> diameters;
  int model = kWhiteBearII;
  double esfmt_A = 1.0, esfmt_B = 0.0;
  std::vector<InteractionSpec> interactions;
  int precision = kFP64;
  int batch = 1;  // problems of this shape evaluated together (1..kMaxBatch)
};

class Engine {
 public:
  explicit Engine(const EngineSpec& spec);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // Full evaluation on device data (functionals.hpp:64-95).  A batched
  // engine evaluates B problems: every array holds B problems back to back.
  //   rho   : B*S*N doubles (device), problem-major then species-major
  //   vext  : B*S*N doubles (device) or null (no external field)
  //   mu    : B*S chemical potentials (beta mu units), host
  //   force : B*S*N doubles (device) receives dOmega/drho * dV
  //   scalars: B*kScalarCount doubles (device): F, Omega, F_id, F_ext, F_hs, F_mf, N_s
  void evaluate(const double* rho, const double* vext, const double* mu, double* force, double* scalars,
                cudaStream_t stream);

  // Hessian-vector product of Omega: hv = d(force)/d(rho) . v (S*N device
  // doubles each); exact, by forward-over-reverse differentiation.  Batch 1 only.
  void hvp(const double* rho, const double* v, const double* mu, double* hv, cudaStream_t stream);
  // Products at one density for several directions (any batch B):
  // hvp_set_point runs the forward pipeline of rho (S*N device doubles) once
  // for every problem slot; hvp_apply then maps B directions v (B*S*N) to B
  // products hv, each direction in its own problem slot of the batched
  // launches.  An evaluate() in between invalidates the point (hvp_apply
  // throws until it is set again).
  void hvp_set_point(const double* rho, cudaStream_t stream);
  void hvp_apply(const double* v, double* hv, cudaStream_t stream);

  const EvalParams& params() const { return p_; }
  int species() const { return p_.S; }
  int batch() const { return p_.batch; }
  long long points() const { return p_.N; }
  long long modes() const { return p_.Nk; }
  int precision() const { return precision_; }
  // Transform path: the fused plane/column kernels (mixed precision on the
  // grids fused.cu specialises: nx and ny, nz in {16, 32, 64, 128}; on by
  // default there) or cuFFT plans with separate k-space kernels.
  bool fusable() const { return fusable_; }
  bool fused() const { return fused_; }
  void set_fused(bool on);
  double a_vdw(int m) const { return a_vdw_[m]; }
  // This library's kernel launches per evaluation (aligned buffers): fused
  // path rho planes, column pass, chunks_ x (channel planes, pointwise,
  // derivative planes), column pass, force planes; the cuFFT paths count
  // their own kernels only.
  // Plane chunks of the fused path's middle stages (1..kMaxChunks, dividing
  // nx); std::invalid_argument otherwise or without the fused path.
  static constexpr int kMaxChunks = 8;
  void set_chunks(int k);
  // Autotuner: times every plane-chunk count (1, 2, 4, 8 dividing nx) on
  // the caller's state, `reps` evaluations each after two untimed ones, and
  // keeps the fastest, for this engine and for engines of the same shape
  // created later in this process.  ms[k - 1]: time per evaluation of count
  // k (0 where not tried).  Returns the count chosen (the current one when
  // the engine has no fused path).  Synchronises the stream.
  // The pointwise kernel variants (see pw_variant_) are tuned with the chunk
  // counts: ms[v * kMaxChunks + k - 1]; *variant receives the variant kept.
  // Several species also tune the column tile width (16, 32), and every
  // chunk count k its pointwise spread d (1, 2, 4, 8 up to k):
  // ms[((tile_index * kPointwiseVariants + v) * kMaxChunks + k - 1) * kSpreads + log2 d]
  // (the faster of the two middle plane-pass widths, which is also tuned).
  // *plane (optional) receives the plane width kept.
  static constexpr int kPointwiseVariants = 6;
  static constexpr int kSpreads = 4;
  int autotune(const double* rho, const double* vext, const double* mu, cudaStream_t stream, int reps,
               double* ms, int* variant, int* tile = nullptr, int* spread = nullptr, int* plane = nullptr);
  // Pointwise grid of one plane chunk: the full pointwise grid (pw_grid)
  // divided by d = min(spread, chunks), 0 = the chunk count (each chunk one
  // share).  Larger shares put more warps on one chunk's FP64 work (a
  // chunk's pointwise launch often runs alone); smaller ones leave SM room
  // for the transforms of the other chunks.  1, 2, 4, 8 or 0.
  void set_pw_spread(int d);
  int pw_spread() const { return pw_div_; }
  int pw_chunk_grid(int K) const;
  // Column tile width of the fused path's column passes (16, or 32 for
  // several species where their spectra fit); std::invalid_argument otherwise.
  void set_col_tile(int tq);
  int col_tile() const;
  // Threads per plane CTA of the fused path's two middle plane passes
  // (channels inverse, derivatives forward): 0 RPlane::NT, 1 twice that
  // (RPlane::NT_WIDE, the width of the one-sequence passes).  The autotuner
  // times both.  plane_width() is -1 without the fused path.
  void set_plane_width(int wide);
  int plane_width() const;
  // Pointwise kernel of the TMA path: 0 generic; one species: 1 / 2 sized
  // for 5 / 6 CTAs per SM, 3 the branch-free FP64 path for warps with eta >=
  // 1e-6 everywhere (5 CTAs per SM), 4 the same with two points per thread
  // (3 CTAs per SM), 5 as 4 at 4 CTAs per SM; std::invalid_argument where the
  // variant does not exist.
  void set_pointwise(int v);
  int pointwise() const { return pw_variant_; }
  bool pointwise_one_species() const { return pw1_; }
  int pw_grid() const;
  int chunks() const { return chunks_; }
  // Changes whenever a setter changes what an evaluation launches (transform
  // path, plane chunks, stage timing): a captured graph of an evaluation is
  // valid only for the generation it was captured at.
  unsigned long long generation() const { return generation_; }
  bool stage_timing_on() const { return timing_; }
  int kernels_per_eval() const { return precision_ == 1 ? (fused_ ? 4 + 3 * chunks_ : 6) : 4; }
  // Reads and clears the device error word (synchronises the stream).
  int take_error(cudaStream_t stream);
  // Anchored split (mixed precision): from set_anchor on, every evaluation
  // transforms rho - rho_a in FP32 instead of rho minus the species means,
  // and adds the FP64 channels, derivative channels and back-convolution of
  // the anchor state rho_a point by point (the FP32 round-off then scales
  // with |rho - rho_a| instead of the density's own swing: a solid near a
  // reference state).  `fp64` is an FP64 engine of the same grid, species,
  // model, interactions and batch; rho_a (device, B*S*N) is evaluated by it
  // once here.  Anchored evaluations run the cuFFT transforms and the
  // generic pointwise kernel.  clear_anchor returns to the mean split.
  void set_anchor(Engine& fp64, const double* rho_a, cudaStream_t stream);
  void clear_anchor();
  bool anchored() const { return anchored_; }
  // Programmatic dependent launch between consecutive passes of the fused
  // path (on by default; results are the same either way).
  void set_dependent_launch(bool on);
  bool dependent_launch() const { return pdl_on_; }
  // FP64 engines: after evaluate(), the real-space channels, derivative
  // channels and back-convolution (before dV) of the evaluated state.
  void export_fields(double* chan, double* deriv, double* hs, cudaStream_t stream) const;

  // Stage timing: when on, every evaluate() records CUDA events between its
  // stages on its stream (one set of a ring of kTimingRing sets per
  // evaluation, so timed evaluations still queue back to back); the ring is
  // harvested when full and by take_stage_times.  Durations (kStages of
  // them, in pipeline order):
  //   0 split / FP32 conversion (mixed), 1 r2c rho, 2 k_forward, 3 c2r channels,
  //   4 pointwise, 5 r2c derivatives, 6 k_backward, 7 c2r force, 8 epilogue
  //   (with the final reduction), 9 (empty: the reduction is folded into 8).
  static constexpr int kStages = 10;
  static constexpr int kTimingRing = 64;
  void set_stage_timing(bool on);
  // Accumulated milliseconds per stage and the number of timed evaluations;
  // clears the accumulators.
  long long take_stage_times(double* ms);
  // Scratch bytes held beyond inputs and outputs.
  size_t scratch_bytes() const { return scratch_bytes_; }

  // Staging buffers of the host-pointer API.
  double* host_rho() { return h_rho_; }
  double* host_vext() { return h_vext_; }
  double* host_force() { return h_force_; }
  double* host_scalars() { return h_scalars_; }
  cudaStream_t stream() const { return stream_; }

 private:
  void build_plans();
  template <class F>
  void with_kernels(bool mixed, F&& f) const;
  void upload_mean_field(const EngineSpec& spec);
  void setup_fused();
  void fused_forward(const double* rho, cudaStream_t stream);
  template <typename R>
  void fused_middle(const double* rho, const double* vext, double* force, bool chunked, cudaStream_t stream);
  void fused_backward(double* force, const MuArgs& mu, const FinalArgs& fin, cudaStream_t stream);
  template <typename R, typename C2>
  void run(const double* rho, const double* vext, const double* mu, double* force, double* scalars,
           cudaStream_t stream);
  template <typename R, typename C2>
  void run_hvp_point(const double* rho, cudaStream_t stream);
  template <typename R, typename C2>
  void run_hvp_apply(const double* v, double* hv, cudaStream_t stream);
  bool hvp_ready_ = false;
  template <typename R, typename C2>
  void forward_stage(const double* in, R* chan_out, double* mean_out, cudaStream_t stream,
                     const double* anchor = nullptr);
  template <typename R, typename C2>
  void backward_stage(R* deriv, const double* dbar, double* out, const MuArgs& mu, const FinalArgs& fin,
                      cudaStream_t stream, const double* hs_anc = nullptr);

  EvalParams p_{};
  int precision_ = kFP64;
  int device_ = 0;
  int grid_k_ = 0, grid_pw_ = 0;
  std::vector<double> a_vdw_;

  // FP64 pipeline buffers (the mixed pipeline views them as float storage).
  // Every per-problem buffer holds B problems back to back.
  void* rho_k_ = nullptr;     // B * S * Nk complex
  void* chan_k_ = nullptr;    // B * C * Nk complex
  void* chan_r_ = nullptr;    // B * C * N real
  void* deriv_r_ = nullptr;   // B * D * N real
  void* deriv_k_ = nullptr;   // B * D * Nk complex
  void* force_k_ = nullptr;   // B * S * Nk complex
  void* hs_r_ = nullptr;      // B * S * N real
  void* rho_lo_ = nullptr;    // B * S * N float (mixed precision input copy)
  double* mf_w_ = nullptr;    // M * Nk real (FP64), shared by the batch
  double* mean_ = nullptr;    // B * kMaxSpecies species means (mixed precision)
  double* dbar_ = nullptr;    // B * kMaxChannels derivative-channel constants (mixed precision)
  double* partials_ = nullptr;
  int* err_ = nullptr;        // device error word (set by bounded waits that gave up)
  unsigned* sync_ = nullptr;  // B last-block counters of k_species_mean (zero between launches)
  void* tan_chan_ = nullptr;  // tangent channels of the exact HVP (allocated on first use)
  double* tan_mean_ = nullptr;
  double* tan_dbar_ = nullptr;
  double* tan_in_ = nullptr;  // aligned copies of rho and v
  int grid_tma_ = 0;
  int grid_stream_ = 0;       // streaming kernels (sums, conversion, epilogue)
  int grid_mean_ = 0;         // k_species_mean
  // grid_* are CTAs per problem: a launch has grid_* x B CTAs
  size_t tma_smem_ = 0, tma_smem_v_ = 0;
  bool pw1_ = false;  // one species, <= 2 mean-field channels, mixed: k_pointwise1_tma exists
  // pointwise kernel of the TMA path: 0 generic (k_pointwise_tma), 1 .. 5
  // the one-species kernel k_pointwise1_tma (grid grid_pw1_[v - 1])
  int pw_variant_ = 0;
  int pw_div_ = 0;  // pointwise grid divisor of a plane chunk (0: the chunk count)
  int grid_pw1_[5] = {0, 0, 0, 0, 0};
  size_t tma1_smem_ = 0, tma1_smem_v_ = 0;    // one point per thread
  size_t tma1_smem2_ = 0, tma1_smem2_v_ = 0;  // two points per thread
  template <typename R>
  void launch_pointwise_tma(const R* chan, R* deriv, const PointwiseArgs& a, long long p0, long long pn, int blk0,
                            int nblk, int grid, cudaStream_t st);
  void* fft_work_ = nullptr;
  size_t scratch_bytes_ = 0;

  // fused transform path
  bool fusable_ = false, fused_ = false;
  // The fused path's middle stages (inverse plane pass, pointwise, forward
  // plane pass of the derivatives) depend only on their own x planes: they
  // run as chunks_ chunks of planes, chunk k > 0 on aux_[k - 1], forked from
  // and joined back into the caller's stream, so the FP64 pointwise work of
  // one chunk overlaps the FP32 transforms of another.
  int chunks_ = 1;
  unsigned long long generation_ = 0;
  std::string tune_key_;  // shape key of the autotuner's cache
  void ensure_chunk_streams(int k);
  std::vector<cudaStream_t> aux_;
  cudaEvent_t fork_ev_ = nullptr;
  std::vector<cudaEvent_t> join_ev_;
  FusedPlan plan_{};
  void* tw_ = nullptr;
  float* wtab_ = nullptr;    // column-pass weight table ([5 S + M][Nk] floats)
  double* pmean_ = nullptr;  // B * S * nx plane means of rho (fused path)
  FftTables tables_{};

  cufftHandle plan_rho_ = 0, plan_chan_ = 0, plan_deriv_ = 0, plan_force_ = 0;
  bool plans_made_ = false;

  void mark(int i, cudaStream_t stream);
  void harvest_stage_times();
  bool timing_ = false, timing_run_ = false;
  std::vector<cudaEvent_t> stage_ev_;  // kTimingRing sets of kStages + 1
  int ring_used_ = 0;                  // sets recorded and not yet harvested
  double stage_ms_[kStages] = {};
  long long stage_count_ = 0;

  bool anchored_ = false;
  bool pdl_on_ = true;
  double* anc_rho_ = nullptr;  // B*S*N
  double* anc_n_ = nullptr;    // B*n_chan*N
  double* anc_d_ = nullptr;    // B*n_deriv*N
  double* anc_hs_ = nullptr;   // B*S*N
  double* h_rho_ = nullptr;   // device staging for host API
  double* h_vext_ = nullptr;
  double* h_force_ = nullptr;
  double* h_scalars_ = nullptr;
  cudaStream_t stream_ = nullptr;
};

}  // namespace cdft
