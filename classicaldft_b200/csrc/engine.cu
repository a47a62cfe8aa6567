// Engine construction (buffers, cuFFT plans, mean-field weights) and the
// evaluation pipeline of one F[rho] + dF/drho call.
#include "engine.cuh"
#include "eval_kernels.cuh"
#include "fused.cuh"
#include "physics_fn.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>

namespace cdft {

namespace {
// The autotuner's choices per engine shape, for the lifetime of the process.
std::mutex g_tune_mu;
std::map<std::string, int> g_tune_chunks;
std::map<std::string, int> g_tune_variant;
std::map<std::string, int> g_tune_tile;
std::map<std::string, int> g_tune_spread;
std::map<std::string, int> g_tune_plane;
}  // namespace

namespace {

template <typename T>
T* dalloc(size_t count, size_t& total) {
  void* p = nullptr;
  if (count == 0) return nullptr;
  CDFT_CUDA(cudaMalloc(&p, count * sizeof(T)));
  total += count * sizeof(T);
  return static_cast<T*>(p);
}

template <typename K>
int occupancy_grid(K kernel, int block, int sms, long long work) {
  int per_sm = 0;
  CDFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0));
  per_sm = std::max(per_sm, 1);
  long long want = (work + block - 1) / block;
  long long g = std::min<long long>((long long)sms * per_sm, want);
  return (int)std::max<long long>(g, 1);
}

__global__ void k_real_part(const double2* __restrict__ in, double* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i].x;
}

// mean_field.hpp:146-196 up to its FFT, one thread per cell: the cell weight
// at the cell's signed offset (zero beyond the cut-off plus half a cell
// diagonal) times dV / N, and per block the sum of weight * dV.
constexpr int kMfThreads = 256;

__global__ void __launch_bounds__(kMfThreads) k_mf_weight(Potential pot, int split, int scheme, double kT, double dx,
                                                          int nx, int ny, int nz, double* __restrict__ out,
                                                          double* __restrict__ partials) {
  const long long N = (long long)nx * ny * nz;
  const double dv = dx * dx * dx;
  const double inv_n = 1.0 / static_cast<double>(N);
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const long iz = (long)(i % nz);
    const long long t = i / nz;
    const long iy = (long)(t % ny);
    const long ix = (long)(t / ny);
    const long sx = phys::signed_offset(ix, nx), sy = phys::signed_offset(iy, ny), sz = phys::signed_offset(iz, nz);
    if (phys::cell_skipped(pot, dx, sx, sy, sz)) {
      out[i] = 0.0;
      continue;
    }
    const double w = phys::cell_weight(pot, split, scheme, kT, dx, sx, sy, sz);
    out[i] = w * dv * inv_n;
    s += w * dv;
  }
  __shared__ double sh[kMfThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < kMfThreads / 32; ++w) b += sh[w];
    partials[blockIdx.x] = b;
  }
}

// a_vdw = the partials summed in a fixed order (deterministic).
__global__ void k_sum_partials(const double* __restrict__ partials, int n, double* __restrict__ out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) s += partials[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *out = s;
}

}  // namespace

// Calls f(model, multi, real-type) with compile-time constants matching this
// engine's FMT model, species count and storage precision.
template <class F>
void Engine::with_kernels(bool mixed, F&& f) const {
  auto by_model = [&](auto multi_c, auto r_c) {
    switch (p_.model) {
      case kRosenfeld: f(std::integral_constant<int, kRosenfeld>{}, multi_c, r_c); break;
      case kRSLT: f(std::integral_constant<int, kRSLT>{}, multi_c, r_c); break;
      case kWhiteBearI: f(std::integral_constant<int, kWhiteBearI>{}, multi_c, r_c); break;
      case kWhiteBearII: f(std::integral_constant<int, kWhiteBearII>{}, multi_c, r_c); break;
      default: f(std::integral_constant<int, kEsFMT>{}, multi_c, r_c); break;
    }
  };
  auto by_multi = [&](auto r_c) {
    if (p_.L.multi)
      by_model(std::true_type{}, r_c);
    else
      by_model(std::false_type{}, r_c);
  };
  if (mixed)
    by_multi(std::type_identity<float>{});
  else
    by_multi(std::type_identity<double>{});
}

namespace {
// f(IC<m>) for a mean-field channel count m in 0..2 of the one-species kernel.
template <class F>
void with_nmf(int m, F&& f) {
  if (m == 0)
    f(std::integral_constant<int, 0>{});
  else if (m == 1)
    f(std::integral_constant<int, 1>{});
  else
    f(std::integral_constant<int, 2>{});
}
}  // namespace

// The TMA-staged pointwise kernel over points p0 .. p0 + pn of every problem:
// the one-species specialisation where it applies, else the generic kernel.
template <typename R>
void Engine::launch_pointwise_tma(const R* chan, R* deriv, const PointwiseArgs& a, long long p0, long long pn,
                                  int blk0, int nblk, int grid, cudaStream_t st) {
  const EvalParams& p = p_;
  const bool vext = a.vext != nullptr;
  const dim3 g(grid, p.batch);
  if constexpr (std::is_same_v<R, float>) {
    if (pw1_ && pw_variant_ > 0 && !a.n_anc) {
      with_kernels(true, [&](auto model_c, auto, auto) {
        constexpr int MD = decltype(model_c)::value;
        with_nmf(p.M, [&](auto nc) {
          constexpr int NMF = decltype(nc)::value;
          const int v = pw_variant_;
          const size_t smem = v >= 4 ? (vext ? tma1_smem2_v_ : tma1_smem2_) : (vext ? tma1_smem_v_ : tma1_smem_);
          // (stream predecessor: the chunk's channel plane pass)
          auto go = [&](auto kern) {
            launch_k(kern, g, dim3(kTmaTile), smem, st, plan_.pdl, p, chan, deriv, a, err_, p0, pn, blk0, nblk);
          };
          if (vext) {
            if (v == 1) go(k_pointwise1_tma<MD, NMF, true, 5>);
            else if (v == 2) go(k_pointwise1_tma<MD, NMF, true, 6>);
            else if (v == 3) go(k_pointwise1_tma<MD, NMF, true, 5, 1, true>);
            else if (v == 4) go(k_pointwise1_tma<MD, NMF, true, 3, 2, true>);
            else go(k_pointwise1_tma<MD, NMF, true, 4, 2, true>);
          } else {
            if (v == 1) go(k_pointwise1_tma<MD, NMF, false, 5>);
            else if (v == 2) go(k_pointwise1_tma<MD, NMF, false, 6>);
            else if (v == 3) go(k_pointwise1_tma<MD, NMF, false, 5, 1, true>);
            else if (v == 4) go(k_pointwise1_tma<MD, NMF, false, 3, 2, true>);
            else go(k_pointwise1_tma<MD, NMF, false, 4, 2, true>);
          }
        });
      });
      CDFT_CUDA(cudaGetLastError());
      return;
    }
  }
  with_kernels(sizeof(R) == sizeof(float), [&](auto model_c, auto multi_c, auto r_c) {
    constexpr int MD = decltype(model_c)::value;
    constexpr bool MU = decltype(multi_c)::value;
    using RT = typename decltype(r_c)::type;
    if constexpr (std::is_same_v<RT, R>)
      k_pointwise_tma<MD, MU, RT><<<g, kTmaTile, vext ? tma_smem_v_ : tma_smem_, st>>>(p, chan, deriv, a, err_, p0,
                                                                                       pn, blk0, nblk);
  });
  CDFT_CUDA(cudaGetLastError());
}

Engine::Engine(const EngineSpec& spec) {
  for (int d = 0; d < 3; ++d)
    if (spec.shape[d] <= 0) throw Error(-1, "Engine: grid dimensions must be positive");
  if (!(spec.dx > 0.0)) throw Error(-1, "Engine: dx must be positive");
  const int S = (int)spec.diameters.size();
  if (S < 1 || S > kMaxSpecies) throw Error(-1, "Engine: number of species must be in [1, 4]");
  for (double d : spec.diameters)
    if (!(d > 0.0)) throw Error(-1, "Engine: hard-sphere diameters must be positive");
  if (spec.model < kRosenfeld || spec.model > kEsFMT) throw Error(-1, "Engine: unknown FMT model id");
  if ((int)spec.interactions.size() > kMaxInteractions) throw Error(-1, "Engine: too many interactions (max 8)");
  if (spec.precision != kFP64 && spec.precision != kMixed) throw Error(-1, "Engine: unknown precision mode");
  if (spec.batch < 1 || spec.batch > kMaxBatch) throw Error(-1, "Engine: batch must be in [1, 64]");
  precision_ = spec.precision;
  CDFT_CUDA(cudaGetDevice(&device_));

  EvalParams& p = p_;
  p.nx = (int)spec.shape[0];
  p.ny = (int)spec.shape[1];
  p.nz = (int)spec.shape[2];
  p.nzh = p.nz / 2 + 1;
  p.N = (long long)p.nx * p.ny * p.nz;
  p.Nk = (long long)p.nx * p.ny * p.nzh;
  p.dx = spec.dx;
  p.dv = spec.dx * spec.dx * spec.dx;
  p.inv_n = 1.0 / (double)p.N;
  p.dkx = 2.0 * kPi / ((double)p.nx * spec.dx);
  p.dky = 2.0 * kPi / ((double)p.ny * spec.dx);
  p.dkz = 2.0 * kPi / ((double)p.nz * spec.dx);
  p.S = S;
  for (int s = 0; s < kMaxSpecies; ++s) {
    const double R = s < S ? 0.5 * spec.diameters[s] : 0.5;
    p.R[s] = R;
    p.inv4piR[s] = 1.0 / (4.0 * kPi * R);
    p.inv4piR2[s] = 1.0 / (4.0 * kPi * R * R);
  }
  p.model = spec.model;
  p.A = spec.esfmt_A;
  p.B = spec.esfmt_B;
  const bool tensor = (p.model == kWhiteBearI || p.model == kWhiteBearII || p.model == kEsFMT);
  p.L = ChannelLayout::make(S > 1, tensor);
  p.M = (int)spec.interactions.size();
  int ch = p.L.n_fmt;
  for (int m = 0; m < p.M; ++m) {
    const auto& it = spec.interactions[m];
    if (it.species_i < 0 || it.species_i >= S || it.species_j < 0 || it.species_j >= S)
      throw Error(-1, "Engine: interaction species index out of range");
    if (it.on_device) {
      if (!(it.kT > 0.0)) throw Error(-1, "Engine: the temperature must be positive");
      if (!(it.potential.sigma > 0.0)) throw Error(-1, "Engine: potential sigma must be positive");
      if (it.scheme < kWeightZero || it.scheme > kWeightGaussF) throw Error(-1, "Engine: unknown weight scheme");
      if (it.split != kWeeksChandlerAndersen && it.split != kBarkerHenderson)
        throw Error(-1, "Engine: unknown split scheme");
    } else if ((long long)it.weight_real.size() != p.N) {
      throw Error(-1, "Engine: interaction weight must have N = nx*ny*nz entries");
    }
    p.mf_i[m] = it.species_i;
    p.mf_j[m] = it.species_j;
    p.mf_chan_j[m] = ch++;
    p.mf_chan_i[m] = (it.species_i != it.species_j) ? ch++ : -1;
  }
  p.n_chan = ch;
  p.n_terms = 4 + S;
  p.batch = spec.batch;
  const int B = p.batch;

  int sms = 0;
  CDFT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
  const bool mixed = precision_ == kMixed;
  const size_t cs = mixed ? sizeof(float2) : sizeof(double2);
  const size_t rs = mixed ? sizeof(float) : sizeof(double);
  size_t tot = 0;
  rho_k_ = dalloc<char>(cs * B * S * p.Nk, tot);
  chan_k_ = dalloc<char>(cs * B * p.n_chan * p.Nk, tot);
  chan_r_ = dalloc<char>(rs * B * p.n_chan * p.N, tot);
  deriv_r_ = dalloc<char>(rs * B * p.L.n_deriv * p.N, tot);
  deriv_k_ = dalloc<char>(cs * B * p.L.n_deriv * p.Nk, tot);
  force_k_ = dalloc<char>(cs * B * S * p.Nk, tot);
  hs_r_ = dalloc<char>(rs * B * S * p.N, tot);
  if (mixed) rho_lo_ = dalloc<char>(sizeof(float) * B * S * p.N, tot);
  mf_w_ = dalloc<double>((size_t)std::max(p.M, 1) * p.Nk, tot);
  mean_ = dalloc<double>((size_t)B * kMaxSpecies, tot);
  dbar_ = dalloc<double>((size_t)B * kMaxChannels, tot);

  // grid sizes from occupancy (148 SMs on B200), shared by the B problems:
  // about one wave of CTAs per launch in total
  auto per_problem = [&](long long g) { return (int)std::max<long long>(1, (g + B - 1) / B); };
  auto pick = [&](auto kern, long long work) {
    return per_problem(occupancy_grid(kern, 256, sms, work * B));
  };
  with_kernels(mixed, [&](auto model_c, auto multi_c, auto r_c) {
    constexpr int MD = decltype(model_c)::value;
    constexpr bool MU = decltype(multi_c)::value;
    using RT = typename decltype(r_c)::type;
    using C2 = std::conditional_t<sizeof(RT) == 4, float2, double2>;
    constexpr bool TE = model_has_tensor(MD);
    grid_pw_ = pick(k_pointwise<MD, MU, RT>, p.N);
    grid_k_ = pick(k_forward<MU, TE, C2>, p.Nk);
  });
  // TMA-staged pointwise kernel: dynamic shared memory for the 3-stage ring
  with_kernels(mixed, [&](auto model_c, auto multi_c, auto r_c) {
    constexpr int MD = decltype(model_c)::value;
    constexpr bool MU = decltype(multi_c)::value;
    using RT = typename decltype(r_c)::type;
    constexpr bool TE = model_has_tensor(MD);
    tma_smem_ = (size_t)kTmaStages * tma_stage_bytes<MU, TE, RT>(S, false);
    tma_smem_v_ = (size_t)kTmaStages * tma_stage_bytes<MU, TE, RT>(S, true);
    CDFT_CUDA(cudaFuncSetAttribute(k_pointwise_tma<MD, MU, RT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)tma_smem_v_));
    int per_sm = 0;
    CDFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pointwise_tma<MD, MU, RT>, kTmaTile,
                                                            tma_smem_v_));
    grid_tma_ = per_problem((long long)sms * std::max(per_sm, 1));
  });
  // the one-species mixed-precision specialisation (k_pointwise1_tma)
  pw1_ = mixed && p.S == 1 && p.M <= 2;
  if (pw1_) {
    with_kernels(true, [&](auto model_c, auto, auto) {
      constexpr int MD = decltype(model_c)::value;
      constexpr bool TE = model_has_tensor(MD);
      with_nmf(p.M, [&](auto nc) {
        constexpr int NMF = decltype(nc)::value;
        const int sb = kTmaStages * tma1_stage_bytes<NMF, false, TE>();
        const int sv = kTmaStages * tma1_stage_bytes<NMF, true, TE>();
        const int sb2 = kTmaStages * tma1_stage_bytes<NMF, false, TE, 2>();
        const int sv2 = kTmaStages * tma1_stage_bytes<NMF, true, TE, 2>();
        // the occupancy of the vext form (the larger stages) sizes both forms' grids
        int per[5] = {0, 0, 0, 0, 0};
        auto prep = [&](auto kb, auto kv, int b, int v, int* out) {
          CDFT_CUDA(cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
          CDFT_CUDA(cudaFuncSetAttribute(kv, cudaFuncAttributeMaxDynamicSharedMemorySize, v));
          CDFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, kv, kTmaTile, v));
        };
        prep(k_pointwise1_tma<MD, NMF, false, 5>, k_pointwise1_tma<MD, NMF, true, 5>, sb, sv, &per[0]);
        prep(k_pointwise1_tma<MD, NMF, false, 6>, k_pointwise1_tma<MD, NMF, true, 6>, sb, sv, &per[1]);
        prep(k_pointwise1_tma<MD, NMF, false, 5, 1, true>, k_pointwise1_tma<MD, NMF, true, 5, 1, true>, sb, sv,
             &per[2]);
        prep(k_pointwise1_tma<MD, NMF, false, 3, 2, true>, k_pointwise1_tma<MD, NMF, true, 3, 2, true>, sb2, sv2,
             &per[3]);
        prep(k_pointwise1_tma<MD, NMF, false, 4, 2, true>, k_pointwise1_tma<MD, NMF, true, 4, 2, true>, sb2, sv2,
             &per[4]);
        for (int v = 0; v < 5; ++v) grid_pw1_[v] = per_problem((long long)sms * std::max(per[v], 1));
        tma1_smem_ = (size_t)sb;
        tma1_smem_v_ = (size_t)sv;
        tma1_smem2_ = (size_t)sb2;
        tma1_smem2_v_ = (size_t)sv2;
      });
    });
    pw_variant_ = 1;
  }
  grid_stream_ = per_problem(std::max<long long>(1, std::min<long long>((long long)sms * 8, (p.N * B + 255) / 256)));
  // the species mean: four blocks per SM in all (its last block sums the
  // partials, so fewer blocks shorten that tail and the counter's contention)
  grid_mean_ = per_problem(std::max<long long>(1, std::min<long long>((long long)sms * 4, (p.N * B + 255) / 256)));
  // (+8: the pointwise grid rounded up to whole chunks, see fused_middle)
  // (a plane chunk may take the whole pointwise grid: kMaxChunks grids)
  partials_ = dalloc<double>(
      (size_t)B *
          ((size_t)std::max({grid_pw_, grid_tma_, grid_stream_, grid_pw1_[0], grid_pw1_[1], grid_pw1_[2],
                             grid_pw1_[3], grid_pw1_[4]}) * kMaxChunks + 8) *
          p.n_terms,
      tot);
  err_ = dalloc<int>(1, tot);
  CDFT_CUDA(cudaMemset(err_, 0, sizeof(int)));
  sync_ = dalloc<unsigned>((size_t)B, tot);
  CDFT_CUDA(cudaMemset(sync_, 0, sizeof(unsigned) * B));

  build_plans();
  upload_mean_field(spec);
  setup_fused();
  scratch_bytes_ = tot;

  CDFT_CUDA(cudaMalloc(&h_rho_, sizeof(double) * B * S * p.N));
  CDFT_CUDA(cudaMalloc(&h_vext_, sizeof(double) * B * S * p.N));
  CDFT_CUDA(cudaMalloc(&h_force_, sizeof(double) * B * S * p.N));
  CDFT_CUDA(cudaMalloc(&h_scalars_, sizeof(double) * B * kScalarCount));
  CDFT_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
}

Engine::~Engine() {
  if (plans_made_) {
    cufftDestroy(plan_rho_);
    cufftDestroy(plan_chan_);
    cufftDestroy(plan_deriv_);
    cufftDestroy(plan_force_);
  }
  for (void* q : {rho_k_, chan_k_, chan_r_, deriv_r_, deriv_k_, force_k_, hs_r_, rho_lo_, (void*)mf_w_,
                  (void*)mean_, (void*)dbar_, (void*)err_, (void*)sync_, tan_chan_, (void*)tan_mean_, (void*)tan_dbar_,
                  (void*)tan_in_,
                  (void*)partials_, fft_work_, tw_, (void*)wtab_, (void*)pmean_, (void*)h_rho_, (void*)h_vext_, (void*)h_force_, (void*)h_scalars_,
                  (void*)anc_rho_, (void*)anc_n_, (void*)anc_d_, (void*)anc_hs_})
    if (q) cudaFree(q);
  if (stream_) cudaStreamDestroy(stream_);
  for (cudaStream_t st : aux_) cudaStreamDestroy(st);
  for (cudaEvent_t ev : join_ev_) cudaEventDestroy(ev);
  if (fork_ev_) cudaEventDestroy(fork_ev_);
  for (cudaEvent_t e : stage_ev_)
    if (e) cudaEventDestroy(e);
}

void Engine::set_stage_timing(bool on) {
  if (on && stage_ev_.empty()) {
    stage_ev_.assign((size_t)kTimingRing * (kStages + 1), nullptr);
    for (cudaEvent_t& e : stage_ev_) CDFT_CUDA(cudaEventCreate(&e));
  }
  if (!on) harvest_stage_times();
  if (on != timing_) ++generation_;
  timing_ = on;
}

void Engine::mark(int i, cudaStream_t stream) {
  if (timing_run_) CDFT_CUDA(cudaEventRecord(stage_ev_[(size_t)ring_used_ * (kStages + 1) + i], stream));
}

// Waits for the recorded sets and adds their stage durations.
void Engine::harvest_stage_times() {
  for (int r = 0; r < ring_used_; ++r) {
    cudaEvent_t* ev = &stage_ev_[(size_t)r * (kStages + 1)];
    CDFT_CUDA(cudaEventSynchronize(ev[kStages]));
    for (int i = 0; i < kStages; ++i) {
      float ms = 0.0f;
      CDFT_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      stage_ms_[i] += ms;
    }
    ++stage_count_;
  }
  ring_used_ = 0;
}

long long Engine::take_stage_times(double* ms) {
  harvest_stage_times();
  for (int i = 0; i < kStages; ++i) {
    ms[i] = stage_ms_[i];
    stage_ms_[i] = 0.0;
  }
  const long long n = stage_count_;
  stage_count_ = 0;
  return n;
}

// The fused transform path (fused.cu) serves mixed-precision engines on the
// grids it has specialisations for; everything else (and the HVP) uses the
// cuFFT plans.
void Engine::setup_fused() {
  const EvalParams& p = p_;
  // shape key of the autotuner's cache: grid, species, batch, model,
  // interactions, precision (and the pointwise variant kept for it)
  tune_key_ = std::to_string(p.nx) + "x" + std::to_string(p.ny) + "x" + std::to_string(p.nz) + " S" +
              std::to_string(p.S) + " B" + std::to_string(p.batch) + " m" + std::to_string(p.model) + " M" +
              std::to_string(p.M) + " P" + std::to_string(precision_);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const auto iv = g_tune_variant.find(tune_key_);
    if (iv != g_tune_variant.end() && (iv->second == 0 || pw1_)) pw_variant_ = iv->second;
    const auto is = g_tune_spread.find(tune_key_);
    if (is != g_tune_spread.end()) pw_div_ = is->second;
  }
  fusable_ = false;
  if (precision_ != kMixed || !fused_plan(p, &plan_)) return;
  // twiddle tables, FP64-rounded
  std::vector<fft::cpx> tw;
  auto table = [&](int M) {
    for (int n = 0; n < M; ++n) {
      const double a = -2.0 * kPi * (double)n / (double)M;
      tw.push_back({(float)std::cos(a), (float)std::sin(a)});
    }
  };
  table(p.nx);
  table(p.ny);
  table(p.nz / 2);
  table(p.nz);
  CDFT_CUDA(cudaMalloc(&tw_, sizeof(fft::cpx) * tw.size()));
  CDFT_CUDA(cudaMemcpy(tw_, tw.data(), sizeof(fft::cpx) * tw.size(), cudaMemcpyHostToDevice));
  const fft::cpx* t = static_cast<const fft::cpx*>(tw_);
  tables_ = FftTables{t, t + p.nx, t + p.nx + p.ny, t + p.nx + p.ny + p.nz / 2};
  CDFT_CUDA(cudaMalloc(&wtab_, sizeof(float) * fused_weight_table_floats(p)));
  CDFT_CUDA(cudaMalloc(&pmean_, sizeof(double) * (size_t)p.batch * p.S * p.nx));
  fused_build_weights(p, mf_w_, wtab_, nullptr);
  CDFT_CUDA(cudaDeviceSynchronize());
  fusable_ = true;
  fused_ = true;
  chunks_ = (p.nx >= 64) ? 4 : 1;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const auto it = g_tune_chunks.find(tune_key_);
    if (it != g_tune_chunks.end()) chunks_ = it->second;
    const auto tt = g_tune_tile.find(tune_key_);
    if (tt != g_tune_tile.end()) fused_plan_set_tile(p, &plan_, tt->second);
    const auto tp = g_tune_plane.find(tune_key_);
    if (tp != g_tune_plane.end()) plan_.plane_wide = tp->second != 0;
  }
  ensure_chunk_streams(chunks_);
}

// Streams and events for k chunks (chunk 0 runs on the caller's stream).
void Engine::ensure_chunk_streams(int k) {
  while ((int)aux_.size() < k - 1) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    CDFT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CDFT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    aux_.push_back(st);
    join_ev_.push_back(ev);
  }
  if (k > 1 && !fork_ev_) CDFT_CUDA(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
}

// Every (plane-chunk count, pointwise variant) pair the engine has, timed on
// the caller's state; the fastest is kept and cached for the shape.
int Engine::autotune(const double* rho, const double* vext, const double* mu, cudaStream_t stream, int reps,
                     double* ms, int* variant, int* tile, int* spread, int* plane) {
  constexpr int kTiles = 2;  // column tile widths 16, 32
  if (ms)
    for (int k = 0; k < kPointwiseVariants * kMaxChunks * kTiles * kSpreads; ++k) ms[k] = 0.0;
  if (variant) *variant = pw_variant_;
  if (tile) *tile = col_tile();
  if (spread) *spread = pw_div_;
  if (plane) *plane = plane_width();
  const bool tune_chunks = fusable_ && fused_;
  const bool tune_tiles = tune_chunks && p_.S > 1;
  if (!tune_chunks && !pw1_) return chunks_;
  if (!rho) throw std::invalid_argument("autotune: rho is required");
  reps = std::max(reps, 1);
  std::vector<double> mu0((size_t)p_.batch * p_.S, 0.0);
  if (!mu) mu = mu0.data();
  const bool timing_was = timing_;
  timing_ = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CDFT_CUDA(cudaEventCreate(&e0));
  CDFT_CUDA(cudaEventCreate(&e1));
  // engines without a tile choice time their current tile (row 0 of the
  // table where they have no fused path)
  const int tile_now = col_tile() == 32 ? 32 : 16;
  int best = chunks_, best_v = pw_variant_, best_t = col_tile(), best_d = pw_div_, best_w = plane_width();
  double best_ms = 0.0;
  for (int wi = 0; wi < (tune_chunks ? 2 : 1); ++wi) {
    if (tune_chunks) set_plane_width(wi);
    for (int ti = 0; ti < kTiles; ++ti) {
      const int tq = 16 << ti;
      if (tune_tiles) {
        if (!fused_plan_set_tile(p_, &plan_, tq)) continue;
        ++generation_;
      } else if (tq != tile_now) {
        continue;
      }
      for (int v = 0; v < kPointwiseVariants; ++v) {
        if (v > 0 && !pw1_) break;
        set_pointwise(v);
        for (int k = 1; k <= kMaxChunks; k *= 2) {
          if (tune_chunks) {
            if (p_.nx % k != 0) continue;
            set_chunks(k);
          } else if (k != chunks_) {
            continue;
          }
          for (int di = 0; di < kSpreads; ++di) {
            const int d = 1 << di;
            if (d > k || (!tune_chunks && d > 1)) break;
            set_pw_spread(d);
            for (int w = 0; w < 2; ++w) evaluate(rho, vext, mu, h_force_, h_scalars_, stream);
            CDFT_CUDA(cudaEventRecord(e0, stream));
            for (int r = 0; r < reps; ++r) evaluate(rho, vext, mu, h_force_, h_scalars_, stream);
            CDFT_CUDA(cudaEventRecord(e1, stream));
            CDFT_CUDA(cudaEventSynchronize(e1));
            float t = 0.0f;
            CDFT_CUDA(cudaEventElapsedTime(&t, e0, e1));
            const double per = (double)t / reps;
            if (ms) {
              double& slot = ms[((ti * kPointwiseVariants + v) * kMaxChunks + k - 1) * kSpreads + di];
              if (slot == 0.0 || per < slot) slot = per;
            }
            if (best_ms == 0.0 || per < best_ms) {
              best_ms = per;
              best = k;
              best_v = v;
              best_d = d;
              if (tune_tiles) best_t = tq;
              if (tune_chunks) best_w = wi;
            }
          }
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  timing_ = timing_was;
  if (tune_tiles) set_col_tile(best_t);
  if (tune_chunks) set_plane_width(best_w);
  if (tune_chunks) set_chunks(best);
  set_pointwise(best_v);
  set_pw_spread(best_d);
  if (variant) *variant = best_v;
  if (tile) *tile = col_tile();
  if (spread) *spread = pw_div_;
  if (plane) *plane = plane_width();
  std::lock_guard<std::mutex> lock(g_tune_mu);
  if (tune_chunks) g_tune_chunks[tune_key_] = best;
  if (tune_chunks) g_tune_plane[tune_key_] = best_w;
  if (tune_tiles) g_tune_tile[tune_key_] = best_t;
  g_tune_variant[tune_key_] = best_v;
  g_tune_spread[tune_key_] = best_d;
  return chunks_;
}

void Engine::set_col_tile(int tq) {
  if (!fusable_) throw std::invalid_argument("column tile: the engine has no fused path");
  const int old = plan_.tq;
  if (!fused_plan_set_tile(p_, &plan_, tq))
    throw std::invalid_argument("column tile: 16 (any engine) or 32 (several species, where the spectra fit)");
  if (plan_.tq != old) ++generation_;
}

int Engine::col_tile() const { return fusable_ ? plan_.tq : 0; }

void Engine::set_plane_width(int wide) {
  if (!fusable_) throw std::invalid_argument("plane width: the engine has no fused path");
  if (wide != 0 && wide != 1) throw std::invalid_argument("plane width: 0 (RPlane::NT threads) or 1 (twice that)");
  if (plan_.plane_wide != (wide == 1)) ++generation_;
  plan_.plane_wide = wide == 1;
}

int Engine::plane_width() const { return fusable_ ? (plan_.plane_wide ? 1 : 0) : -1; }

void Engine::set_pointwise(int v) {
  if (v < 0 || v >= kPointwiseVariants) throw std::invalid_argument("pointwise variant: 0 .. 5");
  if (v > 0 && !pw1_)
    throw std::invalid_argument("pointwise variant: the one-species kernel needs a mixed-precision engine with one "
                                "species and at most two interactions");
  if (v != pw_variant_) ++generation_;
  pw_variant_ = v;
}

int Engine::pw_grid() const { return (pw1_ && pw_variant_ > 0) ? grid_pw1_[pw_variant_ - 1] : grid_tma_; }

int Engine::pw_chunk_grid(int K) const {
  const int d = pw_div_ == 0 ? K : std::min(pw_div_, K);
  return (pw_grid() + d - 1) / d;
}

void Engine::set_pw_spread(int d) {
  if (d != 0 && d != 1 && d != 2 && d != 4 && d != 8)
    throw std::invalid_argument("pointwise spread: 1, 2, 4, 8 or 0 (the chunk count)");
  if (d != pw_div_) ++generation_;
  pw_div_ = d;
}

void Engine::set_chunks(int k) {
  if (!fusable_) throw std::invalid_argument("plane chunks: the engine has no fused path");
  if (k < 1 || k > kMaxChunks || p_.nx % k != 0)
    throw std::invalid_argument("plane chunks: 1..8 dividing nx");
  ensure_chunk_streams(k);
  if (k != chunks_) ++generation_;
  chunks_ = k;
}

void Engine::set_fused(bool on) {
  if (on && !fusable_)
    throw Error(-1, "fused transforms need a mixed-precision engine whose nx, ny, nz are each 16, 32, 48, 64, 96 or "
                    "128 and whose (y, z) plane fits in shared memory");
  if (on != fused_) ++generation_;
  fused_ = on;
}

void Engine::build_plans() {
  const EvalParams& p = p_;
  const bool mixed = precision_ == kMixed;
  long long n[3] = {p.nx, p.ny, p.nz};
  size_t ws[4] = {0, 0, 0, 0};
  cufftHandle* hs[4] = {&plan_rho_, &plan_chan_, &plan_deriv_, &plan_force_};
  const int batch[4] = {p.batch * p.S, p.batch * p.n_chan, p.batch * p.L.n_deriv, p.batch * p.S};
  const cufftType fwd = mixed ? CUFFT_R2C : CUFFT_D2Z;
  const cufftType inv = mixed ? CUFFT_C2R : CUFFT_Z2D;
  const cufftType type[4] = {fwd, inv, fwd, inv};
  for (int i = 0; i < 4; ++i) {
    CDFT_CUFFT(cufftCreate(hs[i]));
    CDFT_CUFFT(cufftSetAutoAllocation(*hs[i], 0));
    const bool r2c = (i == 0 || i == 2);
    CDFT_CUFFT(cufftMakePlanMany64(*hs[i], 3, n, nullptr, 1, r2c ? p.N : p.Nk, nullptr, 1, r2c ? p.Nk : p.N,
                                   type[i], batch[i], &ws[i]));
  }
  plans_made_ = true;
  const size_t wmax = std::max(std::max(ws[0], ws[1]), std::max(ws[2], ws[3]));
  if (wmax > 0) {
    CDFT_CUDA(cudaMalloc(&fft_work_, wmax));
    scratch_bytes_ += wmax;
  }
  for (int i = 0; i < 4; ++i) CDFT_CUFFT(cufftSetWorkArea(*hs[i], fft_work_));
}

void Engine::upload_mean_field(const EngineSpec& spec) {
  const EvalParams& p = p_;
  a_vdw_.clear();
  if (p.M == 0) return;
  // FFT the real-space weights once (mean_field.hpp:194) with a temporary
  // FP64 plan; keep the real part (the weight is real and even).
  double* wr = nullptr;
  double2* wk = nullptr;
  double* partials = nullptr;
  int sms = 0, dev = 0;
  CDFT_CUDA(cudaGetDevice(&dev));
  CDFT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int mf_blocks = (int)std::max<long long>(
      1, std::min<long long>((long long)sms * 8, ((long long)p.N + kMfThreads - 1) / kMfThreads));
  CDFT_CUDA(cudaMalloc(&wr, sizeof(double) * p.N));
  CDFT_CUDA(cudaMalloc(&wk, sizeof(double2) * p.Nk));
  CDFT_CUDA(cudaMalloc(&partials, sizeof(double) * (mf_blocks + 1)));
  cufftHandle plan = 0;
  try {
    CDFT_CUFFT(cufftPlan3d(&plan, p.nx, p.ny, p.nz, CUFFT_D2Z));
    for (int m = 0; m < p.M; ++m) {
      const InteractionSpec& is = spec.interactions[m];
      if (is.on_device) {
        k_mf_weight<<<mf_blocks, kMfThreads>>>(is.potential, is.split, is.scheme, is.kT, p.dx, p.nx, p.ny, p.nz, wr,
                                               partials);
        k_sum_partials<<<1, 32>>>(partials, mf_blocks, partials + mf_blocks);
        CDFT_CUDA(cudaGetLastError());
        double a = 0.0;
        CDFT_CUDA(cudaMemcpy(&a, partials + mf_blocks, sizeof(double), cudaMemcpyDeviceToHost));
        a_vdw_.push_back(a);
      } else {
        CDFT_CUDA(cudaMemcpy(wr, is.weight_real.data(), sizeof(double) * p.N, cudaMemcpyHostToDevice));
        a_vdw_.push_back(is.a_vdw);
      }
      CDFT_CUFFT(cufftExecD2Z(plan, wr, wk));
      k_real_part<<<256, 256>>>(wk, mf_w_ + m * p.Nk, p.Nk);
      CDFT_CUDA(cudaGetLastError());
    }
    CDFT_CUDA(cudaDeviceSynchronize());
  } catch (...) {
    if (plan) cufftDestroy(plan);
    cudaFree(wr);
    cudaFree(wk);
    cudaFree(partials);
    throw;
  }
  cufftDestroy(plan);
  cudaFree(wr);
  cudaFree(wk);
  cudaFree(partials);
}

// Stages 1-3: the weighted-density channels of the field `in` (S*N
// doubles) in real space.  Mixed precision transforms in - mean in FP32 and
// stores the species means in `mean_out`.
template <typename R, typename C2>
void Engine::forward_stage(const double* in, R* chan_out, double* mean_out, cudaStream_t stream,
                           const double* anchor) {
  const EvalParams& p = p_;
  constexpr bool mixed = sizeof(R) == sizeof(float);
  C2* rho_k = static_cast<C2*>(rho_k_);
  C2* chan_k = static_cast<C2*>(chan_k_);
  if constexpr (mixed) {
    const dim3 gs(grid_stream_, p.batch);
    k_species_mean<<<dim3(grid_mean_, p.batch), 256, 0, stream>>>(in, p.N, p.S, partials_, sync_, mean_out);
    k_split_convert<<<gs, 256, 0, stream>>>(in, p.N, p.S, static_cast<float*>(rho_lo_), mean_out, anchor);
    mark(1, stream);
    CDFT_CUFFT(cufftExecR2C(plan_rho_, static_cast<float*>(rho_lo_), reinterpret_cast<cufftComplex*>(rho_k)));
  } else {
    mark(1, stream);
    CDFT_CUFFT(cufftExecD2Z(plan_rho_, const_cast<double*>(in), reinterpret_cast<cufftDoubleComplex*>(rho_k)));
  }
  mark(2, stream);
  const bool multi = p.L.multi, tensor = p.L.tensor;
  const dim3 gk(grid_k_, p.batch);
  if (!multi && !tensor) k_forward<false, false, C2><<<gk, 256, 0, stream>>>(p, rho_k, mf_w_, chan_k);
  if (!multi && tensor) k_forward<false, true, C2><<<gk, 256, 0, stream>>>(p, rho_k, mf_w_, chan_k);
  if (multi && !tensor) k_forward<true, false, C2><<<gk, 256, 0, stream>>>(p, rho_k, mf_w_, chan_k);
  if (multi && tensor) k_forward<true, true, C2><<<gk, 256, 0, stream>>>(p, rho_k, mf_w_, chan_k);
  CDFT_CUDA(cudaGetLastError());
  mark(3, stream);
  if constexpr (mixed)
    CDFT_CUFFT(cufftExecC2R(plan_chan_, reinterpret_cast<cufftComplex*>(chan_k), reinterpret_cast<float*>(chan_out)));
  else
    CDFT_CUFFT(cufftExecZ2D(plan_chan_, reinterpret_cast<cufftDoubleComplex*>(chan_k),
                            reinterpret_cast<double*>(chan_out)));
  mark(4, stream);
}

// Stages 5-7: out += c2r(sum_c conj(W_c) r2c(deriv_c)) dV - mu dV (+ the
// FP64 constants of the split derivative channels, `dbar`).
template <typename R, typename C2>
void Engine::backward_stage(R* deriv, const double* dbar, double* out, const MuArgs& mu, const FinalArgs& fin,
                            cudaStream_t stream, const double* hs_anc) {
  const EvalParams& p = p_;
  constexpr bool mixed = sizeof(R) == sizeof(float);
  C2* deriv_k = static_cast<C2*>(deriv_k_);
  C2* force_k = static_cast<C2*>(force_k_);
  R* hs_r = static_cast<R*>(hs_r_);
  if constexpr (mixed)
    CDFT_CUFFT(cufftExecR2C(plan_deriv_, reinterpret_cast<float*>(deriv), reinterpret_cast<cufftComplex*>(deriv_k)));
  else
    CDFT_CUFFT(cufftExecD2Z(plan_deriv_, reinterpret_cast<double*>(deriv),
                            reinterpret_cast<cufftDoubleComplex*>(deriv_k)));
  mark(6, stream);
  const bool multi = p.L.multi, tensor = p.L.tensor;
  const dim3 gk(grid_k_, p.batch), gs(grid_stream_, p.batch);
  if (!multi && !tensor) k_backward<false, false, C2><<<gk, 256, 0, stream>>>(p, deriv_k, force_k);
  if (!multi && tensor) k_backward<false, true, C2><<<gk, 256, 0, stream>>>(p, deriv_k, force_k);
  if (multi && !tensor) k_backward<true, false, C2><<<gk, 256, 0, stream>>>(p, deriv_k, force_k);
  if (multi && tensor) k_backward<true, true, C2><<<gk, 256, 0, stream>>>(p, deriv_k, force_k);
  CDFT_CUDA(cudaGetLastError());
  mark(7, stream);
  if constexpr (mixed)
    CDFT_CUFFT(cufftExecC2R(plan_force_, reinterpret_cast<cufftComplex*>(force_k), reinterpret_cast<float*>(hs_r)));
  else
    CDFT_CUFFT(cufftExecZ2D(plan_force_, reinterpret_cast<cufftDoubleComplex*>(force_k),
                            reinterpret_cast<double*>(hs_r)));
  mark(8, stream);
  if (!multi && !tensor) k_epilogue<false, false, R><<<gs, 256, 0, stream>>>(p, hs_r, dbar, out, mu, fin, hs_anc);
  if (!multi && tensor) k_epilogue<false, true, R><<<gs, 256, 0, stream>>>(p, hs_r, dbar, out, mu, fin, hs_anc);
  if (multi && !tensor) k_epilogue<true, false, R><<<gs, 256, 0, stream>>>(p, hs_r, dbar, out, mu, fin, hs_anc);
  if (multi && tensor) k_epilogue<true, true, R><<<gs, 256, 0, stream>>>(p, hs_r, dbar, out, mu, fin, hs_anc);
  CDFT_CUDA(cudaGetLastError());
  mark(9, stream);
}

// Fused transform path, stages 1-3: plane pass of rho (split around the
// plane means), column pass (species means, channel products), inverse
// plane pass of every channel.
void Engine::fused_forward(const double* rho, cudaStream_t stream) {
  const EvalParams& p = p_;
  const dim3 gs(grid_stream_, p.batch);
  mark(1, stream);  // the species means come with the plane and column passes
  fft::cpx* prho = static_cast<fft::cpx*>(rho_k_);
  fft::cpx* q = static_cast<fft::cpx*>(chan_k_);
  fused_plane_fwd_rho(plan_, p, rho, pmean_, prho, err_, tables_, stream);
  mark(2, stream);
  fused_col_fwd(plan_, p, prho, pmean_, mean_, wtab_, q, tables_, stream);
  mark(3, stream);
}

// Fused transform path, stages 4-6 on chunks of x planes: inverse plane pass
// of the channels, the pointwise kernel on those planes' points, forward
// plane pass of their derivatives.  Unchunked, the stage marks separate the
// three (stage timing runs this way).
template <typename R>
void Engine::fused_middle(const double* rho, const double* vext, double* force, bool chunked, cudaStream_t stream) {
  const EvalParams& p = p_;
  const int K = chunked ? chunks_ : 1;
  const int per = p.nx / K;
  const int gk = pw_chunk_grid(K);
  const fft::cpx* q = static_cast<const fft::cpx*>(chan_k_);
  fft::cpx* pd = static_cast<fft::cpx*>(deriv_k_);
  float* chan_r = static_cast<float*>(chan_r_);
  float* deriv_r = static_cast<float*>(deriv_r_);
  PointwiseArgs a;
  a.rho = rho;
  a.vext = vext;
  a.force = force;
  a.partials = partials_;
  a.mf_w = mf_w_;
  a.mean = mean_;
  a.dbar_out = dbar_;
  if (K > 1) {
    CDFT_CUDA(cudaEventRecord(fork_ev_, stream));
    for (int k = 1; k < K; ++k) CDFT_CUDA(cudaStreamWaitEvent(aux_[k - 1], fork_ev_, 0));
  }
  for (int k = 0; k < K; ++k) {
    cudaStream_t st = k == 0 ? stream : aux_[k - 1];
    const int ix0 = k * per;
    fused_plane_inv(plan_, p, q, chan_r, err_, ix0, per, tables_, st);
    if (K == 1) mark(4, st);
    const long long p0 = (long long)ix0 * p.ny * p.nz, pn = (long long)per * p.ny * p.nz;
    launch_pointwise_tma<float>(chan_r, deriv_r, a, p0, pn, k * gk, K * gk, gk, st);
    if (K == 1) mark(5, st);
    fused_plane_fwd_deriv(plan_, p, deriv_r, pd, err_, ix0, per, tables_, st);
  }
  if (K > 1) {
    for (int k = 1; k < K; ++k) {
      CDFT_CUDA(cudaEventRecord(join_ev_[k - 1], aux_[k - 1]));
      CDFT_CUDA(cudaStreamWaitEvent(stream, join_ev_[k - 1], 0));
    }
    mark(4, stream);
    mark(5, stream);
  }
  mark(6, stream);
}

// Fused transform path, stages 5-8: plane pass of every derivative channel,
// column pass with the back-convolution, inverse plane pass with the
// epilogue and the scalars.
void Engine::fused_backward(double* force, const MuArgs& mu, const FinalArgs& fin, cudaStream_t stream) {
  const EvalParams& p = p_;
  fft::cpx* pd = static_cast<fft::cpx*>(deriv_k_);
  fft::cpx* pf = static_cast<fft::cpx*>(force_k_);
  fused_col_bwd(plan_, p, pd, wtab_, pf, tables_, stream);
  mark(7, stream);
  fused_plane_inv_epi(plan_, p, pf, dbar_, force, mu, fin, err_, tables_, stream);
  mark(8, stream);
  mark(9, stream);
}

template <typename R, typename C2>
void Engine::run(const double* rho, const double* vext, const double* mu, double* force, double* scalars,
                 cudaStream_t stream) {
  const EvalParams& p = p_;
  constexpr bool mixed = sizeof(R) == sizeof(float);
  for (cufftHandle h : {plan_rho_, plan_chan_, plan_deriv_, plan_force_}) CDFT_CUFFT(cufftSetStream(h, stream));
  R* chan_r = static_cast<R*>(chan_r_);
  R* deriv_r = static_cast<R*>(deriv_r_);

  // cuFFT needs 16-byte aligned FP64 input: stage a misaligned rho
  if (!mixed && ((uintptr_t)rho % 16 != 0)) {
    CDFT_CUDA(cudaMemcpyAsync(h_rho_, rho, sizeof(double) * p.batch * p.S * p.N, cudaMemcpyDeviceToDevice, stream));
    rho = h_rho_;
  }
  timing_run_ = timing_;
  if (timing_run_ && ring_used_ == kTimingRing) harvest_stage_times();
  plan_.pdl = false;  // set below for the chunked fused path only
  mark(0, stream);
  // an anchored split runs the cuFFT transforms (the fused passes split
  // around the plane means)
  const bool anc = mixed && anchored_;
  const bool fused = mixed && fused_ && !anc;
  // 1-3. weighted densities
  // TMA ring when every segment start is 16-byte aligned (N % 4 == 0 and
  // aligned base pointers); otherwise the register-prefetch variant.
  const bool tma = (p.N % 4 == 0) && ((uintptr_t)rho % 16 == 0) && ((uintptr_t)vext % 16 == 0);
  MuArgs ma;
  for (int b = 0; b < kMaxBatch; ++b)
    for (int s = 0; s < kMaxSpecies; ++s) ma.mu[b][s] = (b < p.batch && s < p.S) ? mu[b * p.S + s] : 0.0;
  if (fused && tma) {
    // programmatic dependent launches between consecutive passes of one
    // stream (captured graphs keep them as programmatic edges), except
    // while stage events sit between them
    plan_.pdl = pdl_on_ && !timing_run_;
    // fused path: stages 4-6 in plane chunks (one chunk while stage timing)
    fused_forward(rho, stream);
    if constexpr (sizeof(R) == sizeof(float)) fused_middle<R>(rho, vext, force, !timing_run_, stream);
    const int K = timing_run_ ? 1 : chunks_;
    FinalArgs fin{partials_, K * pw_chunk_grid(K), err_, scalars};
    fused_backward(force, ma, fin, stream);
    mark(10, stream);
    if (timing_run_) {
      timing_run_ = false;
      ++ring_used_;
    }
    return;
  }
  if (fused) {
    fused_forward(rho, stream);
    fused_plane_inv(plan_, p, static_cast<const fft::cpx*>(chan_k_), static_cast<float*>(chan_r_), err_, 0, p.nx,
                    tables_, stream);
    mark(4, stream);
  } else {
    forward_stage<R, C2>(rho, chan_r, mean_, stream, anc ? anc_rho_ : nullptr);
  }
  // 4. pointwise Phi / dPhi + local terms + reductions
  PointwiseArgs a;
  a.rho = rho;
  a.vext = vext;
  a.force = force;
  a.partials = partials_;
  a.mf_w = mf_w_;
  a.mean = mean_;
  a.dbar_out = dbar_;
  if (anc) {
    a.n_anc = anc_n_;
    a.d_anc = anc_d_;
  }
  // (the one-species kernels have no anchored split: the generic grid)
  const int pw_blocks = tma ? (anc ? grid_tma_ : pw_grid()) : grid_pw_;
  const dim3 gp(grid_pw_, p.batch);
  if (tma) {
    launch_pointwise_tma<R>(chan_r, deriv_r, a, 0, p.N, 0, pw_blocks, pw_blocks, stream);
  } else {
    with_kernels(mixed, [&](auto model_c, auto multi_c, auto r_c) {
      constexpr int MD = decltype(model_c)::value;
      constexpr bool MU = decltype(multi_c)::value;
      using RT = typename decltype(r_c)::type;
      if constexpr (std::is_same_v<RT, R>) k_pointwise<MD, MU, RT><<<gp, 256, 0, stream>>>(p, chan_r, deriv_r, a);
    });
    CDFT_CUDA(cudaGetLastError());
  }
  mark(5, stream);
  // 5-7. back-convolution into the force
  if (fused) {
    fused_plane_fwd_deriv(plan_, p, static_cast<const float*>(deriv_r_), static_cast<fft::cpx*>(deriv_k_), err_, 0,
                          p.nx, tables_, stream);
    mark(6, stream);
  }
  // 8. scalars: block 0 of each problem's epilogue reduces the partials
  FinalArgs fin{partials_, pw_blocks, err_, scalars};
  if (fused)
    fused_backward(force, ma, fin, stream);
  else
    backward_stage<R, C2>(deriv_r, dbar_, force, ma, fin, stream, anc ? anc_hs_ : nullptr);
  mark(10, stream);
  if (timing_run_) {
    timing_run_ = false;
    ++ring_used_;
  }
}

// Exact Hessian-vector product (forward-over-reverse): hv = d(force)/d(rho) . v
// = directional derivative of the force vector along v.  The tangent of the
// weighted densities is the forward pipeline applied to v; the pointwise
// kernel carries it through dPhi with dual numbers; the back-convolution is
// linear.
template <typename R, typename C2>
void Engine::run_hvp_point(const double* rho, cudaStream_t stream) {
  const EvalParams& p = p_;
  const size_t SN = (size_t)p.S * p.N;
  for (cufftHandle h : {plan_rho_, plan_chan_, plan_deriv_, plan_force_}) CDFT_CUFFT(cufftSetStream(h, stream));
  if (!tan_chan_) {
    const size_t rs = sizeof(R);
    CDFT_CUDA(cudaMalloc(&tan_chan_, rs * p.batch * p.n_chan * p.N));
    CDFT_CUDA(cudaMalloc(&tan_mean_, sizeof(double) * p.batch * kMaxSpecies));
    CDFT_CUDA(cudaMalloc(&tan_dbar_, sizeof(double) * p.batch * kMaxChannels));
    CDFT_CUDA(cudaMalloc(&tan_in_, sizeof(double) * 2 * p.batch * SN));
  }
  // every problem slot holds the same density: its channels and (mixed) its
  // species means are computed once here for all the directions of later
  // hvp_apply calls
  for (int b = 0; b < p.batch; ++b)
    CDFT_CUDA(cudaMemcpyAsync(tan_in_ + b * SN, rho, sizeof(double) * SN, cudaMemcpyDeviceToDevice, stream));
  forward_stage<R, C2>(tan_in_, static_cast<R*>(chan_r_), mean_, stream);
  hvp_ready_ = true;
}

template <typename R, typename C2>
void Engine::run_hvp_apply(const double* v, double* hv, cudaStream_t stream) {
  const EvalParams& p = p_;
  constexpr bool mixed = sizeof(R) == sizeof(float);
  const size_t SN = (size_t)p.S * p.N;
  for (cufftHandle h : {plan_rho_, plan_chan_, plan_deriv_, plan_force_}) CDFT_CUFFT(cufftSetStream(h, stream));
  double* rho_al = tan_in_;
  double* v_al = tan_in_ + p.batch * SN;
  CDFT_CUDA(cudaMemcpyAsync(v_al, v, sizeof(double) * p.batch * SN, cudaMemcpyDeviceToDevice, stream));
  R* chan_r = static_cast<R*>(chan_r_);
  R* chan_t = static_cast<R*>(tan_chan_);
  R* deriv_r = static_cast<R*>(deriv_r_);
  forward_stage<R, C2>(v_al, chan_t, tan_mean_, stream);
  HvpArgs a;
  a.rho = rho_al;
  a.v = v_al;
  a.hv = hv;
  a.mf_w = mf_w_;
  a.mean = mean_;
  a.tmean = tan_mean_;
  a.tdbar_out = tan_dbar_;
  with_kernels(mixed, [&](auto model_c, auto multi_c, auto r_c) {
    constexpr int MD = decltype(model_c)::value;
    constexpr bool MU = decltype(multi_c)::value;
    using RT = typename decltype(r_c)::type;
    if constexpr (std::is_same_v<RT, R>)
      k_pointwise_hvp<MD, MU, RT><<<dim3(grid_stream_, p.batch), 128, 0, stream>>>(p, chan_r, chan_t, deriv_r, a);
  });
  CDFT_CUDA(cudaGetLastError());
  MuArgs zero{};  // the Hessian does not depend on mu
  backward_stage<R, C2>(deriv_r, tan_dbar_, hv, zero, FinalArgs{nullptr, 0, nullptr, nullptr}, stream);
}

void Engine::hvp_set_point(const double* rho, cudaStream_t stream) {
  if (!rho) throw Error(-1, "hvp: rho is required");
  if (precision_ == kMixed)
    run_hvp_point<float, float2>(rho, stream);
  else
    run_hvp_point<double, double2>(rho, stream);
}

void Engine::hvp_apply(const double* v, double* hv, cudaStream_t stream) {
  if (!v || !hv) throw Error(-1, "hvp: v and hv are required");
  if (!hvp_ready_) throw Error(-1, "hvp: no point set since the last evaluation (hvp_set_point)");
  if (precision_ == kMixed)
    run_hvp_apply<float, float2>(v, hv, stream);
  else
    run_hvp_apply<double, double2>(v, hv, stream);
}

void Engine::hvp(const double* rho, const double* v, const double* mu, double* hv, cudaStream_t stream) {
  if (!rho || !v || !hv) throw Error(-1, "hvp: rho, v and hv are required");
  if (p_.batch != 1) throw Error(-1, "hvp: needs an engine with batch 1 (hvp_set_point / hvp_apply batch)");
  (void)mu;
  hvp_set_point(rho, stream);
  hvp_apply(v, hv, stream);
}

void Engine::export_fields(double* chan, double* deriv, double* hs, cudaStream_t stream) const {
  if (precision_ == kMixed) throw Error(-1, "export_fields: needs an FP64 engine");
  const EvalParams& p = p_;
  const size_t B = (size_t)p.batch, N = (size_t)p.N;
  CDFT_CUDA(cudaMemcpyAsync(chan, chan_r_, sizeof(double) * B * p.n_chan * N, cudaMemcpyDeviceToDevice, stream));
  CDFT_CUDA(cudaMemcpyAsync(deriv, deriv_r_, sizeof(double) * B * p.L.n_deriv * N, cudaMemcpyDeviceToDevice, stream));
  CDFT_CUDA(cudaMemcpyAsync(hs, hs_r_, sizeof(double) * B * p.S * N, cudaMemcpyDeviceToDevice, stream));
}

void Engine::set_anchor(Engine& fp64, const double* rho_a, cudaStream_t stream) {
  if (precision_ != kMixed) throw Error(-1, "anchor: needs a mixed-precision engine");
  if (fp64.precision_ == kMixed) throw Error(-1, "anchor: the anchor engine must be FP64");
  if (!rho_a) throw Error(-1, "anchor: rho_a is required");
  const EvalParams &p = p_, &q = fp64.p_;
  if (p.nx != q.nx || p.ny != q.ny || p.nz != q.nz || p.S != q.S || p.batch != q.batch || p.model != q.model ||
      p.M != q.M || p.n_chan != q.n_chan || p.L.n_deriv != q.L.n_deriv || p.dx != q.dx)
    throw Error(-1, "anchor: the FP64 engine must have the same grid, species, model, interactions and batch");
  const size_t B = (size_t)p.batch, N = (size_t)p.N;
  if (!anc_rho_) {
    CDFT_CUDA(cudaMalloc(&anc_rho_, sizeof(double) * B * p.S * N));
    CDFT_CUDA(cudaMalloc(&anc_n_, sizeof(double) * B * p.n_chan * N));
    CDFT_CUDA(cudaMalloc(&anc_d_, sizeof(double) * B * p.L.n_deriv * N));
    CDFT_CUDA(cudaMalloc(&anc_hs_, sizeof(double) * B * p.S * N));
  }
  CDFT_CUDA(cudaMemcpyAsync(anc_rho_, rho_a, sizeof(double) * B * p.S * N, cudaMemcpyDeviceToDevice, stream));
  std::vector<double> mu0(B * p.S, 0.0);
  fp64.evaluate(anc_rho_, nullptr, mu0.data(), fp64.h_force_, fp64.h_scalars_, stream);
  fp64.export_fields(anc_n_, anc_d_, anc_hs_, stream);
  if (fp64.take_error(stream)) throw Error(-2, "anchor: the FP64 evaluation of the anchor state failed");
  if (!anchored_) ++generation_;
  anchored_ = true;
}

void Engine::set_dependent_launch(bool on) {
  if (on != pdl_on_) ++generation_;
  pdl_on_ = on;
}

void Engine::clear_anchor() {
  if (anchored_) ++generation_;
  anchored_ = false;
}

int Engine::take_error(cudaStream_t stream) {
  int v = 0;
  CDFT_CUDA(cudaMemcpyAsync(&v, err_, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CDFT_CUDA(cudaStreamSynchronize(stream));
  if (v) CDFT_CUDA(cudaMemsetAsync(err_, 0, sizeof(int), stream));
  return v;
}

void Engine::evaluate(const double* rho, const double* vext, const double* mu, double* force, double* scalars,
                      cudaStream_t stream) {
  if (!rho || !force || !scalars || !mu) throw Error(-1, "evaluate: rho, mu, force and scalars are required");
  hvp_ready_ = false;  // the channel buffers are the evaluation's
  if (precision_ == kMixed)
    run<float, float2>(rho, vext, mu, force, scalars, stream);
  else
    run<double, double2>(rho, vext, mu, force, scalars, stream);
}

}  // namespace cdft
