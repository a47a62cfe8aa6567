// Device kernels of one F[rho] + dF/drho evaluation.
//
// Stage map (reference file:line -> kernel):
//   rho_k = r2c(rho)                         hard_sphere.hpp:276-282   cuFFT
//   channels = W(k) rho_k  (+ MF w rho_j)    hard_sphere.hpp:50-67,
//                                            mean_field.hpp:259,275    k_forward
//   n_alpha(r) = c2r(channels)               convolution.hpp:13-26     cuFFT (batched)
//   Phi, dPhi, ideal/external/MF pointwise   hard_sphere.hpp:174-224,
//                                            ideal_gas.hpp:18-37,
//                                            external_field.hpp:16-30,
//                                            mean_field.hpp:261-277    k_pointwise
//   D_k = r2c(dPhi channels)                 convolution.hpp:31-49     cuFFT (batched)
//   F_s(k) = sum_c conj(W_cs(k)) D_c(k)      hard_sphere.hpp:103-136   k_backward
//   force_s += c2r(F_s) dV                   hard_sphere.hpp:250-253   cuFFT + k_epilogue
//   F, Omega                                 functionals.hpp:64-95     k_epilogue (block 0)
//
// W_cs(k) is generated analytically from |k| (weights.hpp:91-137) instead of
// being read from stored tables, and the k-space products of all channels
// (and species) are fused into one pass over k.
//
// Hermitian projection.  The parity-odd vector weights and the off-diagonal
// tensor weights are not Hermitian on the Nyquist lines (the Nyquist index
// maps to +k, grid.hpp:53,55), so the c2r input is not the half-spectrum of a
// real field there.  FFTW's rank>=2 c2r (and pocketfft's) compute the exact
// inverse DFT of its Hermitian projection: on the self-conjugate planes
// kz = 0 and kz = nz/2, X'(kx,ky) = (X(kx,ky) + conj(X(-kx,-ky)))/2.  The
// kernels write X' (through the symmetrised weight of chan_weight_sym), so the
// c2r input is Hermitian and the result does not depend on how a library
// treats non-Hermitian input.
//
// Batched engines.  B problems of one shape are stored back to back
// ([B][channel][N] in real space, [B][channel][Nk] in k-space, so cuFFT
// transforms all B x channels in one plan); every kernel takes its problem
// index from blockIdx.y and offsets its pointers by it.
//
// Mixed precision (FP32 storage, R = float).  The FFTs see only fluctuations:
// rho_s = c_s + delta_rho_s with c_s the exact FP64 mean, and each derivative
// channel D_c = dbar_c + delta_D_c with dbar_c = dPhi/dn_c of the uniform
// fluid at the means.  The constants are convolved exactly in FP64 (a
// constant times the k = 0 weight); only the fluctuations pass through FP32.
#pragma once

#include "cdft_common.cuh"
#include "fmt_models.cuh"

namespace cdft {

// Compile-time channel layout (see ChannelLayout).
template <bool MULTI, bool TENSOR>
struct Lay {
  static constexpr int ETA = 0;
  static constexpr int N2 = 1;
  static constexpr int N1 = MULTI ? 2 : -1;
  static constexpr int N0 = MULTI ? 3 : -1;
  static constexpr int V1 = MULTI ? 4 : 2;
  static constexpr int V0 = MULTI ? 7 : -1;
  static constexpr int T = MULTI ? 10 : 5;  // xx, xy, xz, yy, yz
  static constexpr int NFMT = MULTI ? (TENSOR ? 15 : 10) : (TENSOR ? 10 : 5);
  // Channels whose weight vanishes at k = 0 (the vectors and the off-diagonal
  // tensor components): their split offset and their derivative constant at
  // the mean state are exactly zero (chan_dc; dPhi/dv and dPhi/dT_ij, i != j,
  // vanish where v = 0 and T is diagonal).
  static constexpr bool zero_dc(int c) {
    return (c >= V1 && c < V1 + 3) || (MULTI && c >= V0 && c < V0 + 3) ||
           (TENSOR && (c == T + 1 || c == T + 2 || c == T + 4));
  }
};

// |k|-only factors of the FMT weights of one species at one wavevector.
template <typename T>
struct KWT {
  T w3, w2, fv, A, B;
};
using KW = KWT<double>;

// weights.hpp:91-137: |k|-only factors of the FMT weights of a sphere of radius R.
__device__ inline KW weight_kernels(double k, double R) {
  KW w;
  if (k < 1e-12) {
    w.w3 = (4.0 * kPi / 3.0) * R * R * R;
    w.w2 = 4.0 * kPi * R * R;
    w.fv = 0.0;
    w.A = 0.0;
    w.B = (4.0 * kPi / 3.0) * R * R;
    return w;
  }
  const double kR = k * R;
  double s, c;
  sincos(kR, &s, &c);
  const double ik = 1.0 / k;
  const double ik2 = ik * ik;
  const double ik3 = ik2 * ik;
  const double R2 = R * R;
  w.w3 = 4.0 * kPi * (s - kR * c) * ik3;
  w.w2 = 4.0 * kPi * R * s * ik;
  w.fv = -4.0 * kPi * (R * c - s * ik) * ik2;
  const double gp_over_k = 4.0 * kPi * R * (R * c * ik2 - s * ik3);
  const double gpp = 4.0 * kPi * R * (-R2 * s * ik - 2.0 * R * c * ik2 + 2.0 * s * ik3);
  w.A = -(gpp - gp_over_k) / R2;
  w.B = -gp_over_k / R2;
  return w;
}

// Tensor channel t in 0..4 -> (i, j): xx, xy, xz, yy, yz.
__host__ __device__ constexpr int tchan_i(int t) { return t < 3 ? 0 : 1; }
__host__ __device__ constexpr int tchan_j(int t) { return t < 3 ? t : t - 2; }

// Weight of channel c for species s (times 1/N): the channel is W*rho_s if
// !odd, or i*W*rho_s if odd.  Mirrors weights.hpp:163-179 and the Rosenfeld
// scalings of hard_sphere.hpp:80-85.  c is a compile-time constant at every
// call site (fully unrolled loops), so the branches fold away.
// T = double on the cuFFT path; T = float in the fused column pass (the
// mixed path's FP32 k-space).
template <bool MULTI, bool TENSOR, typename T = double>
__device__ __forceinline__ T chan_weight(int c, int s, const EvalParams& p, const T kk[3], T inv_k2,
                                         const KWT<T>& w, bool& odd) {
  using L = Lay<MULTI, TENSOR>;
  const T in = (T)p.inv_n;
  odd = false;
  if (c == L::ETA) return w.w3 * in;
  if (c == L::N2) return w.w2 * in;
  if (MULTI && c == L::N1) return (w.w2 * in) * (T)p.inv4piR[s];
  if (MULTI && c == L::N0) return (w.w2 * in) * (T)p.inv4piR2[s];
  if (c >= L::V1 && c < L::V1 + 3) {
    odd = true;
    return kk[c - L::V1] * w.fv * in;
  }
  if (MULTI && c >= L::V0 && c < L::V0 + 3) {
    odd = true;
    return (kk[c - L::V0] * w.fv * in) * (T)p.inv4piR[s];
  }
  const int t = c - L::T;
  const int i = tchan_i(t), j = tchan_j(t);
  const T d = (i == j) ? T(1) : T(0);
  return (w.A * kk[i] * kk[j] * inv_k2 + w.B * d) * in;
}

// k = 0 value of channel c for species s without the 1/N (the real-space
// integral of the weight): the constant a uniform unit density produces.
template <bool MULTI, bool TENSOR>
__device__ __forceinline__ double chan_dc(int c, int s, const EvalParams& p) {
  using L = Lay<MULTI, TENSOR>;
  const double R = p.R[s];
  if (c == L::ETA) return (4.0 * kPi / 3.0) * R * R * R;
  if (c == L::N2) return 4.0 * kPi * R * R;
  if (MULTI && c == L::N1) return (4.0 * kPi * R * R) * p.inv4piR[s];
  if (MULTI && c == L::N0) return (4.0 * kPi * R * R) * p.inv4piR2[s];
  if (TENSOR && (c == L::T || c == L::T + 3)) return (4.0 * kPi / 3.0) * R * R;
  return 0.0;
}

__device__ __forceinline__ void k_components(const EvalParams& p, int ix, int iy, int iz, double kk[3]) {
  kk[0] = p.dkx * (double)(ix <= p.nx / 2 ? ix : ix - p.nx);
  kk[1] = p.dky * (double)(iy <= p.ny / 2 ? iy : iy - p.ny);
  kk[2] = p.dkz * (double)iz;
}

template <typename C2>
__device__ __forceinline__ double2 ld2(const C2* a, long long i) {
  C2 v = a[i];
  return make_double2((double)v.x, (double)v.y);
}
template <typename C2>
__device__ __forceinline__ void st2(C2* a, long long i, double2 v);
template <>
__device__ __forceinline__ void st2<double2>(double2* a, long long i, double2 v) { a[i] = v; }
template <>
__device__ __forceinline__ void st2<float2>(float2* a, long long i, double2 v) {
  a[i] = make_float2((float)v.x, (float)v.y);
}

// Channel weight at kk, Hermitian-symmetrised on the self-conjugate planes:
// W'(k) = (W(k) + conj(W(k_m)))/2 with k_m the stored mirror wavevector
// (same |k|).  Since rho_k (and every derivative spectrum) is Hermitian,
// W'(k) rho_k(k) equals the projection (X(k) + conj(X(k_m)))/2 of X = W rho_k
// up to round-off, without reading the mirror mode.  For an odd channel
// (W = i w) the coefficient of i is (w(k) - w(k_m))/2.
template <bool MULTI, bool TENSOR, typename T = double>
__device__ __forceinline__ T chan_weight_sym(int c, int s, const EvalParams& p, const T kk[3], const T km[3],
                                             bool proj, T inv_k2, const KWT<T>& w, bool& odd) {
  T v = chan_weight<MULTI, TENSOR, T>(c, s, p, kk, inv_k2, w, odd);
  if (proj) {
    const T vm = chan_weight<MULTI, TENSOR, T>(c, s, p, km, inv_k2, w, odd);
    v = odd ? T(0.5) * (v - vm) : T(0.5) * (v + vm);
  }
  return v;
}

// One forward channel value at wavevector kk from the species spectra r[]
// (V2 = double2 or float2, matching T).
template <bool MULTI, bool TENSOR, typename T = double, typename V2 = double2>
__device__ __forceinline__ V2 fwd_value(int c, const EvalParams& p, const T kk[3], const T km[3], bool proj,
                                        T inv_k2, const KWT<T>* kw, const V2* r) {
  V2 acc{};
#pragma unroll
  for (int s = 0; s < (MULTI ? kMaxSpecies : 1); ++s) {
    if (s < p.S) {
      bool odd;
      const T w = chan_weight_sym<MULTI, TENSOR, T>(c, s, p, kk, km, proj, inv_k2, kw[s], odd);
      if (odd) {
        acc.x += -w * r[s].y;
        acc.y += w * r[s].x;
      } else {
        acc.x += w * r[s].x;
        acc.y += w * r[s].y;
      }
    }
  }
  return acc;
}

struct KIndex {
  int ix, iy, iz;
  bool proj;
};

__device__ __forceinline__ KIndex decode_k(const EvalParams& p, long long idx) {
  KIndex q;
  q.iz = (int)(idx % p.nzh);
  const long long t = idx / p.nzh;
  q.iy = (int)(t % p.ny);
  q.ix = (int)(t / p.ny);
  q.proj = (q.iz == 0) || (((p.nz & 1) == 0) && q.iz == p.nz / 2);
  return q;
}

// k, 1/k^2 and (on the self-conjugate planes) the mirror wavevector.
__device__ __forceinline__ void k_setup(const EvalParams& p, const KIndex& q, double kk[3], double km[3], double& k,
                                        double& inv_k2) {
  k_components(p, q.ix, q.iy, q.iz, kk);
  const double k2 = kk[0] * kk[0] + kk[1] * kk[1] + kk[2] * kk[2];
  k = sqrt(k2);
  inv_k2 = (k > 1e-12) ? 1.0 / k2 : 0.0;
  if (q.proj) {
    k_components(p, (p.nx - q.ix) % p.nx, (p.ny - q.iy) % p.ny, q.iz, km);
  } else {
    km[0] = kk[0];
    km[1] = kk[1];
    km[2] = kk[2];
  }
}

template <bool MULTI, bool TENSOR, typename C2>
__global__ void __launch_bounds__(256) k_forward(EvalParams p, const C2* __restrict__ rho_k,
                                                 const double* __restrict__ mf_w, C2* __restrict__ chan) {
  using L = Lay<MULTI, TENSOR>;
  const long long Nk = p.Nk;
  rho_k += (long long)blockIdx.y * p.S * Nk;
  chan += (long long)blockIdx.y * p.n_chan * Nk;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < Nk;
       idx += (long long)gridDim.x * blockDim.x) {
    const KIndex q = decode_k(p, idx);
    double kk[3], km[3], k, inv_k2;
    k_setup(p, q, kk, km, k, inv_k2);
    KW kw[kMaxSpecies];
    double2 r[kMaxSpecies];
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
      if (s < p.S) {
        kw[s] = weight_kernels(k, p.R[s]);
        r[s] = ld2(rho_k, s * Nk + idx);
      }
    }
#pragma unroll
    for (int c = 0; c < L::NFMT; ++c)
      st2(chan, c * Nk + idx, fwd_value<MULTI, TENSOR>(c, p, kk, km, q.proj, inv_k2, kw, r));
    // mean-field convolution channels (mean_field.hpp:259, 275); the weight is
    // real and even, so it needs no symmetrisation
    for (int m = 0; m < p.M; ++m) {
      const double w = mf_w[m * Nk + idx];
      const double2 rv = ld2(rho_k, p.mf_j[m] * Nk + idx);
      st2(chan, p.mf_chan_j[m] * Nk + idx, make_double2(w * rv.x, w * rv.y));
      if (p.mf_chan_i[m] >= 0) {
        const double2 ri = ld2(rho_k, p.mf_i[m] * Nk + idx);
        st2(chan, p.mf_chan_i[m] * Nk + idx, make_double2(w * ri.x, w * ri.y));
      }
    }
  }
}

// Back-convolution of species s at kk from the derivative spectra dk[]:
// F_s = sum_c conj(W'_cs) D_c (hard_sphere.hpp:117-134).
template <bool MULTI, bool TENSOR, typename T = double, typename V2 = double2>
__device__ __forceinline__ V2 bwd_value(int s, const EvalParams& p, const T kk[3], const T km[3], bool proj,
                                        T inv_k2, const KWT<T>& w, const V2* d) {
  using L = Lay<MULTI, TENSOR>;
  V2 acc{};
#pragma unroll
  for (int c = 0; c < L::NFMT; ++c) {
    bool odd;
    const T wc = chan_weight_sym<MULTI, TENSOR, T>(c, s, p, kk, km, proj, inv_k2, w, odd);
    if (odd) {  // conj(i w) D = -i w D
      acc.x += wc * d[c].y;
      acc.y += -wc * d[c].x;
    } else {
      acc.x += wc * d[c].x;
      acc.y += wc * d[c].y;
    }
  }
  return acc;
}

template <bool MULTI, bool TENSOR, typename C2>
__global__ void __launch_bounds__(256) k_backward(EvalParams p, const C2* __restrict__ dk, C2* __restrict__ fk) {
  using L = Lay<MULTI, TENSOR>;
  const long long Nk = p.Nk;
  dk += (long long)blockIdx.y * p.L.n_deriv * Nk;
  fk += (long long)blockIdx.y * p.S * Nk;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < Nk;
       idx += (long long)gridDim.x * blockDim.x) {
    const KIndex q = decode_k(p, idx);
    double kk[3], km[3], k, inv_k2;
    k_setup(p, q, kk, km, k, inv_k2);
    double2 d[L::NFMT];
#pragma unroll
    for (int c = 0; c < L::NFMT; ++c) d[c] = ld2(dk, c * Nk + idx);
#pragma unroll
    for (int s = 0; s < (MULTI ? kMaxSpecies : 1); ++s) {
      if (s < p.S) {
        const KW w = weight_kernels(k, p.R[s]);
        st2(fk, s * Nk + idx, bwd_value<MULTI, TENSOR>(s, p, kk, km, q.proj, inv_k2, w, d));
      }
    }
  }
}

// ----------------------------------------------------------- reductions

template <int NT>
__device__ __forceinline__ void block_reduce_store(double (&acc)[NT], int n_terms, double* __restrict__ partials) {
  __shared__ double sh[32][NT];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    double v = acc[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp][t] = v;
  }
  __syncthreads();
  if (threadIdx.x < n_terms) {
    double v = 0.0;
    const int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; ++w) v += sh[w][threadIdx.x];
    partials[blockIdx.x * (long long)n_terms + threadIdx.x] = v;
  }
}

// Sum of `n` partials (stride `stride`, offset `off`) by one warp, fixed order.
__device__ __forceinline__ double warp_sum_partials(const double* __restrict__ partials, int n, int stride, int off) {
  const int lane = threadIdx.x & 31;
  double v = 0.0;
  for (int b = lane; b < n; b += 32) v += partials[b * (long long)stride + off];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return __shfl_sync(0xffffffffu, v, 0);
}

// Sum of `n` partials by the whole block (every thread takes a strided
// share, then a fixed-order tree), so the latency is that of a few loads
// rather than n / 32 dependent ones; the result goes to every thread.  CG:
// L2 loads, for partials written by other blocks of the running grid (the
// caller has fenced).  Call from every thread of the block.
template <bool CG>
__device__ __forceinline__ double block_sum_partials(const double* partials, int n, int stride, int off) {
  __shared__ double sh[32];
  __shared__ double total;
  double v = 0.0;
  for (int b = threadIdx.x; b < n; b += blockDim.x) {
    const double* q = partials + b * (long long)stride + off;
    v += CG ? __ldcg(q) : *q;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    double u = lane < nw ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) u += __shfl_down_sync(0xffffffffu, u, o);
    if (lane == 0) total = u;
  }
  __syncthreads();
  const double r = total;
  __syncthreads();  // sh / total free for the next call
  return r;
}

// True in the one block of problem blockIdx.y that finishes last: every
// block has stored (and fenced) its partials by then.  The threads below
// `writers` stored this block's partials and fence them.  The counter
// returns to zero for the next launch.
__device__ __forceinline__ bool last_block_done(unsigned* counter, int writers) {
  __shared__ bool last;
  if (threadIdx.x < writers) __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned prev = atomicAdd(counter, 1u);
    last = (prev == gridDim.x - 1);
    if (last) *counter = 0u;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Mixed precision, step 1: each species' mean density.  Per-block sums, then
// the last block to finish sums the partials (fixed order) into mean_out.
static __global__ void __launch_bounds__(256) k_species_mean(const double* __restrict__ rho, long long N, int S,
                                                      double* __restrict__ partials, unsigned* __restrict__ counters,
                                                      double* __restrict__ mean_out) {
  rho += (long long)blockIdx.y * S * N;
  partials += (long long)blockIdx.y * gridDim.x * S;
  mean_out += blockIdx.y * kMaxSpecies;
  double acc[kMaxSpecies] = {0.0, 0.0, 0.0, 0.0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long first = blockIdx.x * (long long)blockDim.x + threadIdx.x;
#pragma unroll
  for (int s = 0; s < kMaxSpecies; ++s) {
    if (s >= S) break;
    const double* r = rho + s * N;
    double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    long long i = first;
    for (; i + 7 * stride < N; i += 8 * stride) {  // eight independent loads in flight
#pragma unroll
      for (int u = 0; u < 8; ++u) a[u] += r[i + u * stride];
    }
    for (; i < N; i += stride) a[0] += r[i];
    acc[s] = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
  }
  block_reduce_store<kMaxSpecies>(acc, S, partials);
  if (last_block_done(counters + blockIdx.y, S)) {
    for (int s = 0; s < S; ++s) {
      const double v = block_sum_partials<true>(partials, gridDim.x, S, s);
      if (threadIdx.x == 0) mean_out[s] = v / (double)N;
    }
  }
}

// Mixed precision, step 2: delta_rho = rho - mean in FP32, or with an
// anchor state rho_a (B*S*N, FP64) delta_rho = rho - rho_a.
static __global__ void __launch_bounds__(256) k_split_convert(const double* __restrict__ rho, long long N, int S,
                                                       float* __restrict__ out, const double* __restrict__ mean,
                                                       const double* __restrict__ anchor = nullptr) {
  rho += (long long)blockIdx.y * S * N;
  out += (long long)blockIdx.y * S * N;
  mean += blockIdx.y * kMaxSpecies;
  if (anchor) {
    anchor += (long long)blockIdx.y * S * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
      for (int s = 0; s < S; ++s) out[s * N + i] = (float)(rho[s * N + i] - anchor[s * N + i]);
    return;
  }
  __shared__ double sm[kMaxSpecies];
  if (threadIdx.x < S) sm[threadIdx.x] = mean[threadIdx.x];
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s)
      if (s < S) out[s * N + i] = (float)(rho[s * N + i] - sm[s]);
}

// ------------------------------------------------------------ pointwise

struct PointwiseArgs {
  const double* rho;      // B*S*N
  const double* vext;     // B*S*N or null
  double* force;          // B*S*N: local terms (without -mu dV) written here
  double* partials;       // B * gridDim.x * n_terms
  const double* mf_w;     // M*Nk (k = 0 entries give the mean-field DC weights)
  const double* mean;     // B*kMaxSpecies species means (mixed precision) or null
  double* dbar_out;       // B*kMaxChannels derivative-channel constants (mixed precision) or null
  // anchored split (mixed precision, generic kernels): the FP64 channels
  // (B*n_chan*N) and derivative channels (B*n_deriv*N) of the anchor state
  // replace the constant offsets and dbar point by point; null otherwise
  const double* n_anc = nullptr;
  const double* d_anc = nullptr;
};

// The arguments of problem b of a batch.
__device__ __forceinline__ PointwiseArgs batch_slice(const EvalParams& p, PointwiseArgs a, int b) {
  const long long o = (long long)b * p.S * p.N;
  a.rho += o;
  if (a.vext) a.vext += o;
  a.force += o;
  a.partials += (long long)b * gridDim.x * p.n_terms;
  if (a.mean) a.mean += b * kMaxSpecies;
  if (a.dbar_out) a.dbar_out += b * kMaxChannels;
  if (a.n_anc) a.n_anc += (long long)b * p.n_chan * p.N;
  if (a.d_anc) a.d_anc += (long long)b * p.L.n_deriv * p.N;
  return a;
}

// Derivative-channel values at one point from dPhi (the folding of
// hard_sphere.hpp:121,125,131 plus the T_zz trace folding).
template <bool MULTI, bool TENSOR, class T = double>
__device__ __forceinline__ void fold_derivs(const EvalParams& p, const MeasureDerivs<T>& dm, T* D) {
  using L = Lay<MULTI, TENSOR>;
  const T dzz = TENSOR ? dm.d_t[5] : cst<T>(0.0);
  D[L::ETA] = dm.d_eta;
  if (MULTI) {
    D[L::N2] = dm.d_n2 + dzz;
    D[L::N1] = dm.d_n1;
    D[L::N0] = dm.d_n0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      D[L::V1 + c] = dm.d_v1[c];
      D[L::V0 + c] = dm.d_v0[c];
    }
  } else {
    D[L::N2] = dm.d_n2 + dm.d_n1 * p.inv4piR[0] + dm.d_n0 * p.inv4piR2[0] + dzz;
#pragma unroll
    for (int c = 0; c < 3; ++c) D[L::V1 + c] = dm.d_v1[c] + dm.d_v0[c] * p.inv4piR[0];
  }
  if (TENSOR) {
    D[L::T + 0] = dm.d_t[0] - dzz;        // xx
    D[L::T + 1] = 2.0 * dm.d_t[1];        // xy
    D[L::T + 2] = 2.0 * dm.d_t[2];        // xz
    D[L::T + 3] = dm.d_t[3] - dzz;        // yy
    D[L::T + 4] = 2.0 * dm.d_t[4];        // yz
  }
}

// Measures at one point from the channel values n[] (species-summed).
template <bool MULTI, bool TENSOR, class T = double>
__device__ __forceinline__ void assemble(const EvalParams& p, const T* n, Measures<T>& m) {
  using L = Lay<MULTI, TENSOR>;
  m.eta = n[L::ETA];
  m.n2 = n[L::N2];
#pragma unroll
  for (int c = 0; c < 3; ++c) m.v1[c] = n[L::V1 + c];
  if (MULTI) {
    m.n1 = n[L::N1];
    m.n0 = n[L::N0];
#pragma unroll
    for (int c = 0; c < 3; ++c) m.v0[c] = n[L::V0 + c];
  } else {
    m.n1 = m.n2 * p.inv4piR[0];
    m.n0 = m.n2 * p.inv4piR2[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) m.v0[c] = m.v1[c] * p.inv4piR[0];
  }
  if (TENSOR) {
#pragma unroll
    for (int c = 0; c < 5; ++c) m.t[c] = n[L::T + c];
    m.t[5] = m.n2 - m.t[0] - m.t[3];
  } else {
#pragma unroll
    for (int c = 0; c < 6; ++c) m.t[c] = cst<T>(0.0);
  }
}

// Per-block constants of the mixed-precision split: channel offsets (the FP64
// convolution of the species means) and the derivative-channel constants
// dbar (dPhi of the uniform fluid at the means).  Thread 0 fills shared memory.
template <int MODEL, bool MULTI>
__device__ __forceinline__ void split_prologue(const EvalParams& p, const PointwiseArgs& a, double* s_off,
                                               double* s_dbar, bool write_dbar) {
  constexpr bool TENSOR = model_has_tensor(MODEL);
  using L = Lay<MULTI, TENSOR>;
  constexpr int NF = L::NFMT;
  if (threadIdx.x == 0) {
    for (int c = 0; c < p.n_chan; ++c) s_off[c] = 0.0;
#pragma unroll
    for (int c = 0; c < NF; ++c)
      for (int s = 0; s < p.S; ++s) s_off[c] += a.mean[s] * chan_dc<MULTI, TENSOR>(c, s, p);
    for (int m = 0; m < p.M; ++m) {
      const double w0 = a.mf_w[m * p.Nk] * (double)p.N;
      s_off[p.mf_chan_j[m]] = a.mean[p.mf_j[m]] * w0;
      if (p.mf_chan_i[m] >= 0) s_off[p.mf_chan_i[m]] = a.mean[p.mf_i[m]] * w0;
    }
    Measures<double> m0;
    assemble<MULTI, TENSOR>(p, s_off, m0);
    double phi0;
    MeasureDerivs<double> d0;
    double D0[NF];
    if (fmt_phi_dphi<MODEL, double>(p.A, p.B, m0, phi0, d0)) {
      fold_derivs<MULTI, TENSOR>(p, d0, D0);
    } else {
#pragma unroll
      for (int c = 0; c < NF; ++c) D0[c] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < NF; ++c) {
      s_dbar[c] = D0[c];
      if (write_dbar) a.dbar_out[c] = D0[c];
    }
  }
  __syncthreads();
}

// Everything computed at one grid point: Phi and the derivative channels, the
// ideal-gas / external / mean-field local force, and the reduction terms.
// cur[0..NF) are the FMT channel values, cur[NF..NF+n_mf_pre) the first
// mean-field channels (others are read from `chan`).
template <int MODEL, bool MULTI, typename RT, int NPRE>
__device__ __forceinline__ void point_body(const EvalParams& p, const PointwiseArgs& a, const double* cur,
                                           int n_mf_pre, const double* rs, const double* vs, long long idx,
                                           const RT* __restrict__ chan, RT* __restrict__ deriv,
                                           const double* s_off, const double* s_dbar, double* acc) {
  constexpr bool TENSOR = model_has_tensor(MODEL);
  using L = Lay<MULTI, TENSOR>;
  constexpr bool SPLIT = sizeof(RT) == sizeof(float);
  constexpr int NF = L::NFMT;
  const long long N = p.N;
  // the split offsets of channel c at this point: the constants of the
  // species means, or the anchor state's FP64 channels
  const double* na = (SPLIT && a.n_anc) ? a.n_anc + idx : nullptr;
  const double* da = (SPLIT && a.d_anc) ? a.d_anc + idx : nullptr;
  auto off = [&](int c) { return SPLIT ? (na ? na[(long long)c * N] : s_off[c]) : 0.0; };
  double n[NF];
#pragma unroll
  for (int c = 0; c < NF; ++c) n[c] = cur[c] + off(c);
  Measures<double> m;
  double phi = 0.0;
  MeasureDerivs<double> dm;
  double D[NF];
  bool live;
  if constexpr (MULTI) {
    assemble<MULTI, TENSOR>(p, n, m);
    live = fmt_phi_dphi<MODEL, double>(p.A, p.B, m, phi, dm);
    if (live) fold_derivs<MULTI, TENSOR>(p, dm, D);
  } else {
    // one species: n0, n1, v0 are multiples of n2, v1, folded into Phi
    // and its derivatives directly
    using L1 = Lay<false, TENSOR>;
    m.eta = n[L1::ETA];
    m.n2 = n[L1::N2];
#pragma unroll
    for (int c = 0; c < 3; ++c) m.v1[c] = n[L1::V1 + c];
    if constexpr (TENSOR) {
#pragma unroll
      for (int c = 0; c < 5; ++c) m.t[c] = n[L1::T + c];
      m.t[5] = m.n2 - m.t[0] - m.t[3];
    } else {
#pragma unroll
      for (int c = 0; c < 6; ++c) m.t[c] = 0.0;
    }
    live = fmt_phi_dphi<MODEL, double, true>(p.A, p.B, m, phi, dm, p.inv4piR2[0], p.inv4piR[0]);
    if (live) {
      const double dzz = TENSOR ? dm.d_t[5] : 0.0;
      D[L1::ETA] = dm.d_eta;
      D[L1::N2] = dm.d_n2 + dzz;
#pragma unroll
      for (int c = 0; c < 3; ++c) D[L1::V1 + c] = dm.d_v1[c];
      if constexpr (TENSOR) {
        D[L1::T + 0] = dm.d_t[0] - dzz;
        D[L1::T + 1] = 2.0 * dm.d_t[1];
        D[L1::T + 2] = 2.0 * dm.d_t[2];
        D[L1::T + 3] = dm.d_t[3] - dzz;
        D[L1::T + 4] = 2.0 * dm.d_t[4];
      }
    }
  }
  if (!live) {
    phi = 0.0;
#pragma unroll
    for (int c = 0; c < NF; ++c) D[c] = 0.0;
  }
  acc[kTermHS] += phi;
#pragma unroll
  for (int c = 0; c < NF; ++c)
    __stcs(deriv + c * N + idx, (RT)(SPLIT ? D[c] - (da ? da[(long long)c * N] : s_dbar[c]) : D[c]));
  if constexpr (!MULTI) {
    // one species: every interaction is species 0 with itself, channel NF + q
    const double r = rs[0], v = vs[0];
    const double lr = log(r < 1e-300 ? 1e-300 : r);
    acc[kTermId] += r * (lr - 1.0);
    acc[kTermExt] += r * v;
    acc[kTermN0] += r;
    double f0 = lr + v;  // -mu dV is added by k_epilogue
    for (int q = 0; q < p.M; ++q) {
      double cj;
      if (q < n_mf_pre)
        cj = q == 0 ? cur[NF] : cur[NPRE - 1];
      else
        cj = (double)chan[(NF + q) * N + idx];
      cj += off(NF + q);
      acc[kTermMF] += 0.5 * r * cj;
      f0 += cj;
    }
    __stcs(a.force + idx, f0 * p.dv);
  } else {
    double f[kMaxSpecies];
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
      if (s < p.S) {
        const double r = rs[s];
        const double v = vs[s];
        const double lr = log(r < 1e-300 ? 1e-300 : r);
        acc[kTermId] += r * (lr - 1.0);
        acc[kTermExt] += r * v;
        acc[kTermN0 + s] += r;
        f[s] = lr * p.dv + v * p.dv;  // -mu dV is added by k_epilogue
      }
    }
    for (int q = 0; q < p.M; ++q) {
      const int i = p.mf_i[q], j = p.mf_j[q];
      const int cjx = p.mf_chan_j[q];
      const int cix = p.mf_chan_i[q];
      double cj = 0.0, ci = 0.0;
      bool hj = false, hi = false;
#pragma unroll
      for (int c = NF; c < NPRE; ++c) {
        if (c == cjx && c - NF < n_mf_pre) { cj = cur[c]; hj = true; }
        if (c == cix && c - NF < n_mf_pre) { ci = cur[c]; hi = true; }
      }
      if (!hj) cj = (double)chan[cjx * N + idx];
      cj += off(cjx);
      double ri = 0.0;
#pragma unroll
      for (int s = 0; s < kMaxSpecies; ++s)
        if (s == i) ri = rs[s];
      acc[kTermMF] += 0.5 * ri * cj;
      if (i == j) {
#pragma unroll
        for (int s = 0; s < kMaxSpecies; ++s)
          if (s == i) f[s] += cj * p.dv;
      } else {
        if (!hi) ci = (double)chan[cix * N + idx];
        ci += off(cix);
#pragma unroll
        for (int s = 0; s < kMaxSpecies; ++s) {
          if (s == i) f[s] += 0.5 * cj * p.dv;
          if (s == j) f[s] += 0.5 * ci * p.dv;
        }
      }
    }
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s)
      if (s < p.S) __stcs(a.force + s * N + idx, f[s]);
  }
}

// Plain variant (any N): each thread loads the next point's inputs before
// working on the current one.
template <int MODEL, bool MULTI, typename RT>
__global__ void __launch_bounds__(256) k_pointwise(EvalParams p, const RT* __restrict__ chan, RT* __restrict__ deriv,
                                                   PointwiseArgs a_all) {
  constexpr bool TENSOR = model_has_tensor(MODEL);
  using L = Lay<MULTI, TENSOR>;
  constexpr bool SPLIT = sizeof(RT) == sizeof(float);
  constexpr int NT = 4 + (MULTI ? kMaxSpecies : 1);  // the partial sums (one species: 5)
  constexpr int NF = L::NFMT;
  constexpr int NPRE = NF + 2;
  const PointwiseArgs a = batch_slice(p, a_all, blockIdx.y);
  chan += (long long)blockIdx.y * p.n_chan * p.N;
  deriv += (long long)blockIdx.y * p.L.n_deriv * p.N;
  __shared__ double s_off[kMaxChannels];
  __shared__ double s_dbar[NF];
  if (SPLIT) split_prologue<MODEL, MULTI>(p, a, s_off, s_dbar, blockIdx.x == 0);
  const long long N = p.N;
  double acc[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) acc[t] = 0.0;
  const int n_mf_pre = (p.n_chan - NF) < 2 ? (p.n_chan - NF) : 2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N; idx += stride) {
    double cur[NPRE], rs[kMaxSpecies], vs[kMaxSpecies];
#pragma unroll
    for (int q = 0; q < NPRE; ++q)
      if (q < NF || q - NF < n_mf_pre) cur[q] = (double)__ldcs(chan + q * N + idx);
#pragma unroll
    for (int s = 0; s < (MULTI ? kMaxSpecies : 1); ++s) {
      if (s < p.S) {
        rs[s] = __ldcs(a.rho + s * N + idx);
        vs[s] = a.vext ? __ldcs(a.vext + s * N + idx) : 0.0;
      }
    }
    point_body<MODEL, MULTI, RT, NPRE>(p, a, cur, n_mf_pre, rs, vs, idx, chan, deriv, s_off, s_dbar, acc);
  }
  block_reduce_store<NT>(acc, p.n_terms, a.partials);
}

// ---- TMA-staged variant (N % 4 == 0) -----------------------------------
//
// Each CTA walks tiles of kTmaTile points.  Every input segment of a tile
// (channel values, rho, V_ext) streams from HBM into a kTmaStages-deep
// shared-memory ring with cp.async.bulk (TMA bulk copies, no multicast), signalled by an
// mbarrier with transaction counts; each thread then reads its point from
// shared memory.  There is no block-wide barrier per tile: each warp counts
// itself out of a stage when it has read it, and the last warp out issues
// the stage's next fill, so warps run ahead of one another by up to the
// ring depth and the FP64 work of a tile overlaps the loads of the next two.

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Bounded wait: gives up after `limit` polls, so a lost transaction can never
// hang the GPU; the caller records the failure in the engine's error word.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit) {
  for (long long it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

constexpr int kTmaTile = 128;
constexpr int kTmaStages = 3;
constexpr long long kWaitLimit = 1ll << 26;

template <bool MULTI, bool TENSOR, typename RT>
__host__ __device__ constexpr int tma_stage_bytes(int S, bool vext) {
  return (Lay<MULTI, TENSOR>::NFMT + 2) * kTmaTile * (int)sizeof(RT) + S * kTmaTile * 8 * (vext ? 2 : 1);
}

// Points p0 .. p0 + pn - 1 of every problem (p0 a multiple of 4); the
// partial sums of block blockIdx.x go to slot blk0 + blockIdx.x of nblk per
// problem, so launches over disjoint point ranges fill one partials array.
template <int MODEL, bool MULTI, typename RT>
__global__ void __launch_bounds__(kTmaTile, 5) k_pointwise_tma(EvalParams p, const RT* __restrict__ chan,
                                                            RT* __restrict__ deriv, PointwiseArgs a_all,
                                                            int* err, long long p0, long long pn, int blk0,
                                                            int nblk) {
  pdl_trigger();
  pdl_wait();
  constexpr bool TENSOR = model_has_tensor(MODEL);
  using L = Lay<MULTI, TENSOR>;
  constexpr bool SPLIT = sizeof(RT) == sizeof(float);
  constexpr int NT = 4 + (MULTI ? kMaxSpecies : 1);  // the partial sums (one species: 5)
  constexpr int NF = L::NFMT;
  constexpr int NPRE = NF + 2;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bars[kTmaStages];
  __shared__ double s_off[kMaxChannels];
  __shared__ double s_dbar[NF];
  __shared__ int s_fail;
  __shared__ int s_out[kTmaStages];             // warps done with the stage's current fill
  __shared__ long long s_issued[kTmaStages];    // last local tile issued into the stage
  PointwiseArgs a = batch_slice(p, a_all, blockIdx.y);
  a.partials = a_all.partials + ((long long)blockIdx.y * nblk + blk0) * p.n_terms;
  chan += (long long)blockIdx.y * p.n_chan * p.N;
  deriv += (long long)blockIdx.y * p.L.n_deriv * p.N;
  const bool has_v = a.vext != nullptr;
  const int S = p.S;
  const int n_mf_pre = (p.n_chan - NF) < 2 ? (p.n_chan - NF) : 2;
  const int n_in = NF + n_mf_pre;  // channel segments per tile
  const int stage_bytes = NPRE * kTmaTile * (int)sizeof(RT) + S * kTmaTile * 8 * (has_v ? 2 : 1);
  const long long N = p.N;  // the stride of the channel and species arrays
  const long long ntiles = (pn + kTmaTile - 1) / kTmaTile;
  const long long mine = (blockIdx.x < ntiles) ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int st = 0; st < kTmaStages; ++st) {
      mbar_init(&bars[st], 1);
      s_out[st] = 0;
      s_issued[st] = -1;
    }
    s_fail = 0;
    fence_mbar_init();
  }
  if (SPLIT) split_prologue<MODEL, MULTI>(p, a, s_off, s_dbar, blk0 + blockIdx.x == 0);
  __syncthreads();

  auto stage_ptr = [&](int st) { return smem + (size_t)st * stage_bytes; };
  auto issue = [&](long long i) {  // local tile i -> stage i % kTmaStages
    const int st = (int)(i % kTmaStages);
    const long long tile = blockIdx.x + i * gridDim.x;
    const long long start = p0 + tile * kTmaTile;
    const long long cnt = (p0 + pn - start) < kTmaTile ? (p0 + pn - start) : kTmaTile;
    const uint32_t cb = (uint32_t)(cnt * sizeof(RT));
    const uint32_t db = (uint32_t)(cnt * 8);
    unsigned char* base = stage_ptr(st);
    s_issued[st] = i;
    mbar_arrive_expect_tx(&bars[st], cb * n_in + db * S * (has_v ? 2 : 1));
    for (int q = 0; q < n_in; ++q)
      bulk_copy_g2s(base + (size_t)q * kTmaTile * sizeof(RT), chan + q * N + start, cb, &bars[st]);
    unsigned char* rb = base + (size_t)NPRE * kTmaTile * sizeof(RT);
    for (int s = 0; s < S; ++s) bulk_copy_g2s(rb + (size_t)s * kTmaTile * 8, a.rho + s * N + start, db, &bars[st]);
    if (has_v)
      for (int s = 0; s < S; ++s)
        bulk_copy_g2s(rb + (size_t)(S + s) * kTmaTile * 8, a.vext + s * N + start, db, &bars[st]);
  };

  if (tid == 0)
    for (long long i = 0; i < mine && i < kTmaStages; ++i) issue(i);

  double acc[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) acc[t] = 0.0;
  constexpr int kWarps = kTmaTile / 32;
  const int lane = tid & 31;
  volatile int* fail = &s_fail;
  // stage st = i % kTmaStages and its phase parity, advanced per tile
  int st = 0;
  uint32_t par = 0;
  long long idx = p0 + (long long)blockIdx.x * kTmaTile + tid;
  const long long idx_step = (long long)gridDim.x * kTmaTile, idx_end = p0 + pn;
  for (long long i = 0; i < mine; ++i, idx += idx_step) {
    if (*fail) break;
    if (!mbar_wait_bounded(&bars[st], par, kWaitLimit)) {
      *fail = 1;
      break;
    }
    if (idx < idx_end) {
      const RT* cs = reinterpret_cast<const RT*>(stage_ptr(st));
      const double* rb = reinterpret_cast<const double*>(stage_ptr(st) + (size_t)NPRE * kTmaTile * sizeof(RT));
      double cur[NPRE], rs[kMaxSpecies], vs[kMaxSpecies];
#pragma unroll
      for (int q = 0; q < NPRE; ++q)
        if (q < NF || q - NF < n_mf_pre) cur[q] = (double)cs[q * kTmaTile + tid];
#pragma unroll
      for (int s = 0; s < (MULTI ? kMaxSpecies : 1); ++s) {
        if (s < S) {
          rs[s] = rb[s * kTmaTile + tid];
          vs[s] = has_v ? rb[(S + s) * kTmaTile + tid] : 0.0;
        }
      }
      point_body<MODEL, MULTI, RT, NPRE>(p, a, cur, n_mf_pre, rs, vs, idx, chan, deriv, s_off, s_dbar, acc);
    }
    // this warp is done reading stage st; the last warp out refills it
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&s_out[st], 1) == kWarps - 1) {
        s_out[st] = 0;
        if (i + kTmaStages < mine) {
          fence_proxy_async();
          issue(i + kTmaStages);
        }
      }
    }
    if (++st == kTmaStages) {
      st = 0;
      par ^= 1u;
    }
  }
  __syncthreads();
  if (s_fail) {
    // drain the copies still in flight (bounded) before the CTA exits
    if (tid == 0) {
      *err = 1;
      for (int st = 0; st < kTmaStages; ++st)
        if (s_issued[st] >= 0)
          mbar_wait_bounded(&bars[st], (uint32_t)((s_issued[st] / kTmaStages) & 1), kWaitLimit);
    }
    __syncthreads();
  }
  block_reduce_store<NT>(acc, p.n_terms, a.partials);
}

// One species with NMF (0..2) mean-field channels, mixed precision: the TMA
// ring of k_pointwise_tma with every layout size a compile-time constant, no
// species or interaction loops and no runtime channel selection (the common
// case of every benchmark workload).  Same arithmetic as point_body's
// one-species branch, so the results equal the generic kernel's.
//
// PTS points per thread (a tile of PTS * kTmaTile points): the FP64 chains
// of the points are independent, so the scheduler can interleave them.
// FAST: a warp whose points all have eta >= 1e-6 takes the branch-free
// path of fmt_phi_dphi (no Taylor branch, no skip, one reciprocal for
// 1/eta and 1/(1 - eta)); other warps take the exact path.  FAST results
// may differ from the exact path's in the last bit of the FP64 values.
template <int NMF, bool HAS_V, bool TENSOR, int PTS = 1>
__host__ __device__ constexpr int tma1_stage_bytes() {
  return ((Lay<false, TENSOR>::NFMT + NMF) * kTmaTile * 4 + kTmaTile * 8 * (HAS_V ? 2 : 1)) * PTS;
}

// Phi/dPhi and the local terms at one point of the one-species kernel:
// derivative channels minus their split constants out (FP32), the local
// force terms out (FP64), the five partial sums accumulated where `live`.
template <int MODEL, int NMF, bool HAS_V, bool FAST>
__device__ __forceinline__ void pw1_point(const EvalParams& p, const double* n, double r, double v, bool live,
                                          const double* dbar, float* __restrict__ deriv, double* __restrict__ force,
                                          long long idx, long long N, double (&acc)[5]) {
  constexpr bool TENSOR = model_has_tensor(MODEL);
  using L = Lay<false, TENSOR>;
  constexpr int NF = L::NFMT;
  Measures<double> m;
  m.eta = n[L::ETA];
  m.n2 = n[L::N2];
#pragma unroll
  for (int c = 0; c < 3; ++c) m.v1[c] = n[L::V1 + c];
  if constexpr (TENSOR) {
#pragma unroll
    for (int c = 0; c < 5; ++c) m.t[c] = n[L::T + c];
    m.t[5] = m.n2 - m.t[0] - m.t[3];
  } else {
#pragma unroll
    for (int c = 0; c < 6; ++c) m.t[c] = 0.0;
  }
  double phi = 0.0;
  MeasureDerivs<double> dm;
  double D[NF];
  if (fmt_phi_dphi<MODEL, double, true, FAST>(p.A, p.B, m, phi, dm, p.inv4piR2[0], p.inv4piR[0])) {
    const double dzz = TENSOR ? dm.d_t[5] : 0.0;
    D[L::ETA] = dm.d_eta;
    D[L::N2] = dm.d_n2 + dzz;
#pragma unroll
    for (int c = 0; c < 3; ++c) D[L::V1 + c] = dm.d_v1[c];
    if constexpr (TENSOR) {
      D[L::T + 0] = dm.d_t[0] - dzz;
      D[L::T + 1] = 2.0 * dm.d_t[1];
      D[L::T + 2] = 2.0 * dm.d_t[2];
      D[L::T + 3] = dm.d_t[3] - dzz;
      D[L::T + 4] = 2.0 * dm.d_t[4];
    }
  } else {
    phi = 0.0;
#pragma unroll
    for (int c = 0; c < NF; ++c) D[c] = 0.0;
  }
  const double lr = log(r < 1e-300 ? 1e-300 : r);
  double f0 = HAS_V ? lr + v : lr;  // -mu dV is added by k_epilogue
#pragma unroll
  for (int q = 0; q < NMF; ++q) f0 += n[NF + q];
  if (live) {
    acc[kTermHS] += phi;
    // (no subtraction where the constant is zero: fewer shared loads and FP64 adds)
#pragma unroll
    for (int c = 0; c < NF; ++c) __stcs(deriv + c * N + idx, L::zero_dc(c) ? (float)D[c] : (float)(D[c] - dbar[c]));
    acc[kTermId] += r * (lr - 1.0);
    if constexpr (HAS_V) acc[kTermExt] += r * v;
    acc[kTermN0] += r;
#pragma unroll
    for (int q = 0; q < NMF; ++q) acc[kTermMF] += 0.5 * r * n[NF + q];
    __stcs(force + idx, f0 * p.dv);
  }
}

// MINB: the CTAs per SM the register allocation is sized for; the variants
// (PTS, FAST, MINB) are chosen per engine shape by the autotuner.
template <int MODEL, int NMF, bool HAS_V, int MINB, int PTS = 1, bool FAST = false>
__global__ void __launch_bounds__(kTmaTile, MINB) k_pointwise1_tma(EvalParams p, const float* __restrict__ chan,
                                                             float* __restrict__ deriv, PointwiseArgs a_all,
                                                             int* err, long long p0, long long pn, int blk0,
                                                             int nblk) {
  pdl_trigger();
  pdl_wait();
  constexpr bool TENSOR = model_has_tensor(MODEL);
  using L = Lay<false, TENSOR>;
  constexpr int NF = L::NFMT;
  constexpr int NIN = NF + NMF;  // float segments per tile
  constexpr int TP = kTmaTile * PTS;  // points per tile
  constexpr int RHO_OFF = NIN * TP * 4;
  constexpr int V_OFF = RHO_OFF + TP * 8;
  constexpr int STAGE = tma1_stage_bytes<NMF, HAS_V, TENSOR, PTS>();
  constexpr int NT = 5;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bars[kTmaStages];
  __shared__ double s_off[kMaxChannels];
  __shared__ double s_dbar[NF];
  __shared__ int s_fail;
  __shared__ int s_out[kTmaStages];
  __shared__ long long s_issued[kTmaStages];
  PointwiseArgs a = batch_slice(p, a_all, blockIdx.y);
  a.partials = a_all.partials + ((long long)blockIdx.y * nblk + blk0) * p.n_terms;
  chan += (long long)blockIdx.y * p.n_chan * p.N;
  deriv += (long long)blockIdx.y * NF * p.N;
  const long long N = p.N;
  const long long ntiles = (pn + TP - 1) / TP;
  const long long mine = (blockIdx.x < ntiles) ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int st = 0; st < kTmaStages; ++st) {
      mbar_init(&bars[st], 1);
      s_out[st] = 0;
      s_issued[st] = -1;
    }
    s_fail = 0;
    fence_mbar_init();
  }
  split_prologue<MODEL, false>(p, a, s_off, s_dbar, blk0 + blockIdx.x == 0);
  __syncthreads();

  auto issue = [&](long long i) {  // local tile i -> stage i % kTmaStages
    const int st = (int)(i % kTmaStages);
    const long long start = p0 + (blockIdx.x + i * gridDim.x) * TP;
    const long long cnt = (p0 + pn - start) < TP ? (p0 + pn - start) : TP;
    const uint32_t cb = (uint32_t)(cnt * 4), db = (uint32_t)(cnt * 8);
    unsigned char* base = smem + (size_t)st * STAGE;
    s_issued[st] = i;
    mbar_arrive_expect_tx(&bars[st], cb * NIN + db * (HAS_V ? 2 : 1));
#pragma unroll
    for (int q = 0; q < NIN; ++q) bulk_copy_g2s(base + q * TP * 4, chan + q * N + start, cb, &bars[st]);
    bulk_copy_g2s(base + RHO_OFF, a.rho + start, db, &bars[st]);
    if constexpr (HAS_V) bulk_copy_g2s(base + V_OFF, a.vext + start, db, &bars[st]);
  };
  if (tid == 0)
    for (long long i = 0; i < mine && i < kTmaStages; ++i) issue(i);

  // the split offsets stay in shared memory and the model constants in the
  // parameter bank: held in registers they would spill
  const double* off = s_off;
  const double* dbar = s_dbar;
  double acc[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) acc[t] = 0.0;
  constexpr int kWarps = kTmaTile / 32;
  const int lane = tid & 31;
  volatile int* fail = &s_fail;
  int st = 0;
  uint32_t par = 0;
  long long idx = p0 + (long long)blockIdx.x * TP + tid;
  const long long idx_step = (long long)gridDim.x * TP, idx_end = p0 + pn;
  for (long long i = 0; i < mine; ++i, idx += idx_step) {
    // every exit decision is warp-uniform, so the warp stays converged for
    // the vote and the warp barrier below
    if (__any_sync(0xffffffffu, *fail != 0)) break;
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[st], par, kWaitLimit))) {
      *fail = 1;
      break;
    }
    const unsigned char* base = smem + (size_t)st * STAGE;
    double n[PTS][NIN], r[PTS], v[PTS];
    bool live[PTS];
    bool lane_fast = true;
#pragma unroll
    for (int j = 0; j < PTS; ++j) {
      const int o = tid + j * kTmaTile;
      live[j] = idx + j * kTmaTile < idx_end;
      const float* cs = reinterpret_cast<const float*>(base) + o;
#pragma unroll
      for (int c = 0; c < NIN; ++c) {
        const double x = (double)cs[c * TP];
        n[j][c] = (c < NF && L::zero_dc(c)) ? x : x + off[c];
      }
      r[j] = reinterpret_cast<const double*>(base + RHO_OFF)[o];
      v[j] = HAS_V ? reinterpret_cast<const double*>(base + V_OFF)[o] : 0.0;
      lane_fast = lane_fast && (!live[j] || n[j][L::ETA] >= 1e-6);
    }
    if (FAST && __all_sync(0xffffffffu, lane_fast)) {
#pragma unroll
      for (int j = 0; j < PTS; ++j)
        pw1_point<MODEL, NMF, HAS_V, true>(p, n[j], r[j], v[j], live[j], dbar, deriv, a.force,
                                           idx + j * kTmaTile, N, acc);
    } else {
#pragma unroll
      for (int j = 0; j < PTS; ++j)
        if (live[j])
          pw1_point<MODEL, NMF, HAS_V, false>(p, n[j], r[j], v[j], true, dbar, deriv, a.force,
                                              idx + j * kTmaTile, N, acc);
    }
    // this warp is done reading stage st; the last warp out refills it
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&s_out[st], 1) == kWarps - 1) {
        s_out[st] = 0;
        if (i + kTmaStages < mine) {
          fence_proxy_async();
          issue(i + kTmaStages);
        }
      }
    }
    if (++st == kTmaStages) {
      st = 0;
      par ^= 1u;
    }
  }
  __syncthreads();
  if (s_fail) {
    if (tid == 0) {
      *err = 1;
      for (int q = 0; q < kTmaStages; ++q)
        if (s_issued[q] >= 0) mbar_wait_bounded(&bars[q], (uint32_t)((s_issued[q] / kTmaStages) & 1), kWaitLimit);
    }
    __syncthreads();
  }
  block_reduce_store<NT>(acc, p.n_terms, a.partials);
}

// ---- exact Hessian-vector product ---------------------------------------

struct HvpArgs {
  const double* rho;   // S*N
  const double* v;     // S*N direction
  double* hv;          // S*N: local tangent terms written here
  const double* mf_w;
  const double* mean;  // species means of rho (mixed precision)
  const double* tmean; // species means of v (mixed precision)
  double* tdbar_out;   // tangent derivative-channel constants (mixed precision)
};

// Tangent of the pointwise stage along the tangent channels: dual numbers
// through fmt_phi_dphi give the derivative channels' directional derivative
// (forward over the hand-written reverse).  Local terms: the ideal gas
// tangent v / rho dV (zero where the reference clamps rho to 1e-300,
// ideal_gas.hpp:312) and the mean-field convolution of v.
template <int MODEL, bool MULTI, typename RT>
__global__ void __launch_bounds__(128) k_pointwise_hvp(EvalParams p, const RT* __restrict__ chan,
                                                       const RT* __restrict__ tchan, RT* __restrict__ deriv,
                                                       HvpArgs a) {
  constexpr bool TENSOR = model_has_tensor(MODEL);
  using L = Lay<MULTI, TENSOR>;
  constexpr bool SPLIT = sizeof(RT) == sizeof(float);
  constexpr int NF = L::NFMT;
  __shared__ double s_off[kMaxChannels];
  __shared__ double s_toff[kMaxChannels];
  __shared__ double s_tdbar[NF];
  {
    // direction b of a batched product: its own problem slot of every array
    const int b = blockIdx.y;
    const long long cn = (long long)p.n_chan * p.N, sn = (long long)p.S * p.N;
    chan += b * cn;
    tchan += b * cn;
    deriv += b * (long long)p.L.n_deriv * p.N;
    a.rho += b * sn;
    a.v += b * sn;
    a.hv += b * sn;
    a.mean += b * kMaxSpecies;
    a.tmean += b * kMaxSpecies;
    a.tdbar_out += b * kMaxChannels;
  }
  if (SPLIT) {
    if (threadIdx.x == 0) {
      for (int c = 0; c < p.n_chan; ++c) s_off[c] = s_toff[c] = 0.0;
#pragma unroll
      for (int c = 0; c < NF; ++c)
        for (int s = 0; s < p.S; ++s) {
          s_off[c] += a.mean[s] * chan_dc<MULTI, TENSOR>(c, s, p);
          s_toff[c] += a.tmean[s] * chan_dc<MULTI, TENSOR>(c, s, p);
        }
      for (int m = 0; m < p.M; ++m) {
        const double w0 = a.mf_w[m * p.Nk] * (double)p.N;
        s_off[p.mf_chan_j[m]] = a.mean[p.mf_j[m]] * w0;
        s_toff[p.mf_chan_j[m]] = a.tmean[p.mf_j[m]] * w0;
        if (p.mf_chan_i[m] >= 0) {
          s_off[p.mf_chan_i[m]] = a.mean[p.mf_i[m]] * w0;
          s_toff[p.mf_chan_i[m]] = a.tmean[p.mf_i[m]] * w0;
        }
      }
      Dual n0[NF];
#pragma unroll
      for (int c = 0; c < NF; ++c) n0[c] = Dual{s_off[c], s_toff[c]};
      Measures<Dual> m0;
      assemble<MULTI, TENSOR, Dual>(p, n0, m0);
      Dual phi0;
      MeasureDerivs<Dual> d0;
      Dual D0[NF];
      if (fmt_phi_dphi<MODEL, Dual>(p.A, p.B, m0, phi0, d0)) {
        fold_derivs<MULTI, TENSOR, Dual>(p, d0, D0);
      } else {
#pragma unroll
        for (int c = 0; c < NF; ++c) D0[c] = Dual{0.0, 0.0};
      }
#pragma unroll
      for (int c = 0; c < NF; ++c) {
        s_tdbar[c] = D0[c].d;
        if (blockIdx.x == 0) a.tdbar_out[c] = D0[c].d;
      }
    }
    __syncthreads();
  }
  const long long N = p.N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
       idx += (long long)gridDim.x * blockDim.x) {
    Dual n[NF];
#pragma unroll
    for (int c = 0; c < NF; ++c)
      n[c] = Dual{(double)chan[c * N + idx] + (SPLIT ? s_off[c] : 0.0),
                  (double)tchan[c * N + idx] + (SPLIT ? s_toff[c] : 0.0)};
    Measures<Dual> m;
    assemble<MULTI, TENSOR, Dual>(p, n, m);
    Dual phi;
    MeasureDerivs<Dual> dm;
    Dual D[NF];
    if (fmt_phi_dphi<MODEL, Dual>(p.A, p.B, m, phi, dm)) {
      fold_derivs<MULTI, TENSOR, Dual>(p, dm, D);
    } else {
#pragma unroll
      for (int c = 0; c < NF; ++c) D[c] = Dual{0.0, 0.0};
    }
#pragma unroll
    for (int c = 0; c < NF; ++c) deriv[c * N + idx] = (RT)(SPLIT ? D[c].d - s_tdbar[c] : D[c].d);
    double h[kMaxSpecies];
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
      if (s < p.S) {
        const double r = a.rho[s * N + idx];
        h[s] = (r < 1e-300 ? 0.0 : a.v[s * N + idx] / r) * p.dv;
      }
    }
    for (int q = 0; q < p.M; ++q) {
      const int i = p.mf_i[q], j = p.mf_j[q];
      const int cjx = p.mf_chan_j[q];
      const double tj = (double)tchan[cjx * N + idx] + (SPLIT ? s_toff[cjx] : 0.0);
      if (i == j) {
#pragma unroll
        for (int s = 0; s < kMaxSpecies; ++s)
          if (s == i) h[s] += tj * p.dv;
      } else {
        const int cix = p.mf_chan_i[q];
        const double ti = (double)tchan[cix * N + idx] + (SPLIT ? s_toff[cix] : 0.0);
#pragma unroll
        for (int s = 0; s < kMaxSpecies; ++s) {
          if (s == i) h[s] += 0.5 * tj * p.dv;
          if (s == j) h[s] += 0.5 * ti * p.dv;
        }
      }
    }
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s)
      if (s < p.S) a.hv[s * N + idx] = h[s];
  }
}

// Final reduction of one problem: the pointwise kernel's partials into the
// scalar block [F, Omega, F_id, F_ext, F_hs, F_mf, N_0 .. N_{S-1}]
// (functionals.hpp:72-92), fixed summation order, the whole block per term.
__device__ __forceinline__ void reduce_final(const double* __restrict__ partials, int nblocks, const EvalParams& p,
                                             const double* mu, const int* __restrict__ err, double* __restrict__ out) {
  __shared__ double sh[4 + kMaxSpecies];
  const int n_terms = p.n_terms;
  for (int t = 0; t < n_terms; ++t) {
    const double v = block_sum_partials<false>(partials, nblocks, n_terms, t);
    if (threadIdx.x == 0) sh[t] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double dv = p.dv;
    const double f_id = sh[kTermId] * dv;
    const double f_ext = sh[kTermExt] * dv;
    const double f_hs = sh[kTermHS] * dv;
    const double f_mf = sh[kTermMF] * dv;
    double F = 0.0;
    F += f_id;
    F += f_ext;
    F += f_hs;
    if (p.M > 0) F += f_mf;
    double muN = 0.0;
    for (int s = 0; s < p.S; ++s) muN += mu[s] * sh[kTermN0 + s] * dv;
    const bool bad = err && *err != 0;  // a bounded wait gave up: poison the result
    out[0] = bad ? __longlong_as_double(0x7ff8000000000000ll) : F;
    out[1] = bad ? __longlong_as_double(0x7ff8000000000000ll) : F - muN;
    out[2] = f_id;
    out[3] = f_ext;
    out[4] = f_hs;
    out[5] = f_mf;
    for (int s = 0; s < p.S; ++s) out[6 + s] = sh[kTermN0 + s] * dv;
    for (int s = p.S; s < kMaxSpecies; ++s) out[6 + s] = 0.0;  // unused species slots
  }
}

// force_s += c2r(F_s) dV - mu_s dV (+ the FP64 constant of the split
// derivative channels) (hard_sphere.hpp:250-253, ideal_gas.hpp:33).  Block 0
// of each problem also finishes the scalars (the pointwise kernel, which
// wrote the partials, completed before this launch).
template <bool MULTI, bool TENSOR, typename RT>
__global__ void __launch_bounds__(256) k_epilogue(EvalParams p, const RT* __restrict__ hs, const double* __restrict__ dbar,
                                                  double* __restrict__ force, const __grid_constant__ MuArgs mu,
                                                  FinalArgs fin, const double* __restrict__ hs_anc = nullptr) {
  using L = Lay<MULTI, TENSOR>;
  constexpr bool SPLIT = sizeof(RT) == sizeof(float);
  const int b = blockIdx.y;
  const long long N = p.N;
  if (blockIdx.x == 0 && fin.scalars)
    reduce_final(fin.partials + (long long)b * fin.nblocks * p.n_terms, fin.nblocks, p, mu.mu[b], fin.err,
                 fin.scalars + b * kScalarCount);
  hs += (long long)b * p.S * N;
  force += (long long)b * p.S * N;
  dbar += b * kMaxChannels;
  if (hs_anc) {
    // anchored split: the anchor's FP64 back-convolution replaces the
    // constants of the split derivative channels
    hs_anc += (long long)b * p.S * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
      for (int s = 0; s < p.S; ++s)
        force[s * N + i] = force[s * N + i] + ((double)hs[s * N + i] + hs_anc[s * N + i]) * p.dv - mu.mu[b][s] * p.dv;
    return;
  }
  __shared__ double s_const[kMaxSpecies];
  if (threadIdx.x < p.S) {
    const int s = threadIdx.x;
    double v = 0.0;
    if (SPLIT) {
#pragma unroll
      for (int c = 0; c < L::NFMT; ++c) v += chan_dc<MULTI, TENSOR>(c, s, p) * dbar[c];
    }
    s_const[s] = v * p.dv - mu.mu[b][s] * p.dv;
  }
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
      if (s < p.S) force[s * N + i] = force[s * N + i] + (double)hs[s * N + i] * p.dv + s_const[s];
    }
}

}  // namespace cdft
