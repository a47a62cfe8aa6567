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
//   F, Omega                                 functionals.hpp:64-95     k_reduce_final
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
// kernels write X' explicitly, so the c2r input is exactly Hermitian and the
// result does not depend on how a library treats non-Hermitian input.
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
};

struct KW {
  double w3, w2, fv, A, B;
};

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
template <bool MULTI, bool TENSOR>
__device__ __forceinline__ double chan_weight(int c, int s, const EvalParams& p, const double kk[3], double inv_k2,
                                              const KW& w, bool& odd) {
  using L = Lay<MULTI, TENSOR>;
  const double in = p.inv_n;
  odd = false;
  if (c == L::ETA) return w.w3 * in;
  if (c == L::N2) return w.w2 * in;
  if (MULTI && c == L::N1) return (w.w2 * in) * p.inv4piR[s];
  if (MULTI && c == L::N0) return (w.w2 * in) * p.inv4piR2[s];
  if (c >= L::V1 && c < L::V1 + 3) {
    odd = true;
    return kk[c - L::V1] * w.fv * in;
  }
  if (MULTI && c >= L::V0 && c < L::V0 + 3) {
    odd = true;
    return (kk[c - L::V0] * w.fv * in) * p.inv4piR[s];
  }
  const int t = c - L::T;
  const int i = tchan_i(t), j = tchan_j(t);
  const double d = (i == j) ? 1.0 : 0.0;
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

// One forward channel value at wavevector kk from the species spectra r[].
template <bool MULTI, bool TENSOR>
__device__ __forceinline__ double2 fwd_value(int c, const EvalParams& p, const double kk[3], double inv_k2,
                                             const KW* kw, const double2* r) {
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int s = 0; s < (MULTI ? kMaxSpecies : 1); ++s) {
    if (s < p.S) {
      bool odd;
      const double w = chan_weight<MULTI, TENSOR>(c, s, p, kk, inv_k2, kw[s], odd);
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
  long long midx;
};

__device__ __forceinline__ KIndex decode_k(const EvalParams& p, long long idx) {
  KIndex q;
  q.iz = (int)(idx % p.nzh);
  const long long t = idx / p.nzh;
  q.iy = (int)(t % p.ny);
  q.ix = (int)(t / p.ny);
  q.proj = (q.iz == 0) || (((p.nz & 1) == 0) && q.iz == p.nz / 2);
  q.midx = 0;
  if (q.proj) {
    const int mx = (p.nx - q.ix) % p.nx;
    const int my = (p.ny - q.iy) % p.ny;
    q.midx = q.iz + (long long)p.nzh * (my + (long long)p.ny * mx);
  }
  return q;
}

template <bool MULTI, bool TENSOR, typename C2>
__global__ void __launch_bounds__(256) k_forward(EvalParams p, const C2* __restrict__ rho_k,
                                                 const double* __restrict__ mf_w, C2* __restrict__ chan) {
  using L = Lay<MULTI, TENSOR>;
  const long long Nk = p.Nk;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < Nk;
       idx += (long long)gridDim.x * blockDim.x) {
    const KIndex q = decode_k(p, idx);
    double kk[3];
    k_components(p, q.ix, q.iy, q.iz, kk);
    const double k2 = kk[0] * kk[0] + kk[1] * kk[1] + kk[2] * kk[2];
    const double k = sqrt(k2);
    const double inv_k2 = (k > 1e-12) ? 1.0 / k2 : 0.0;
    KW kw[kMaxSpecies];
    double2 r[kMaxSpecies];
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
      if (s < p.S) {
        kw[s] = weight_kernels(k, p.R[s]);
        r[s] = ld2(rho_k, s * Nk + idx);
      }
    }
    double km[3];
    double2 rm[kMaxSpecies];
    if (q.proj) {
      const int mx = (p.nx - q.ix) % p.nx;
      const int my = (p.ny - q.iy) % p.ny;
      k_components(p, mx, my, q.iz, km);
#pragma unroll
      for (int s = 0; s < kMaxSpecies; ++s)
        if (s < p.S) rm[s] = ld2(rho_k, s * Nk + q.midx);
    }
#pragma unroll
    for (int c = 0; c < L::NFMT; ++c) {
      double2 x = fwd_value<MULTI, TENSOR>(c, p, kk, inv_k2, kw, r);
      if (q.proj) {
        const double2 xm = fwd_value<MULTI, TENSOR>(c, p, km, inv_k2, kw, rm);
        x.x = 0.5 * (x.x + xm.x);
        x.y = 0.5 * (x.y - xm.y);
      }
      st2(chan, c * Nk + idx, x);
    }
    // mean-field convolution channels (mean_field.hpp:259, 275)
    for (int m = 0; m < p.M; ++m) {
      const double w = mf_w[m * Nk + idx];
      const double wm = q.proj ? mf_w[m * Nk + q.midx] : w;
      for (int side = 0; side < 2; ++side) {
        const int ch = side == 0 ? p.mf_chan_j[m] : p.mf_chan_i[m];
        if (ch < 0) continue;
        const int sp = side == 0 ? p.mf_j[m] : p.mf_i[m];
        const double2 rv = ld2(rho_k, sp * Nk + idx);
        double2 x = make_double2(w * rv.x, w * rv.y);
        if (q.proj) {
          const double2 rmv = ld2(rho_k, sp * Nk + q.midx);
          x.x = 0.5 * (x.x + wm * rmv.x);
          x.y = 0.5 * (x.y - wm * rmv.y);
        }
        st2(chan, ch * Nk + idx, x);
      }
    }
  }
}

// Back-convolution of species s at kk from the derivative spectra dk[]:
// F_s = sum_c conj(W_cs) D_c (hard_sphere.hpp:117-134).
template <bool MULTI, bool TENSOR>
__device__ __forceinline__ double2 bwd_value(int s, const EvalParams& p, const double kk[3], double inv_k2,
                                             const KW& w, const double2* d) {
  using L = Lay<MULTI, TENSOR>;
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int c = 0; c < L::NFMT; ++c) {
    bool odd;
    const double wc = chan_weight<MULTI, TENSOR>(c, s, p, kk, inv_k2, w, odd);
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
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < Nk;
       idx += (long long)gridDim.x * blockDim.x) {
    const KIndex q = decode_k(p, idx);
    double kk[3];
    k_components(p, q.ix, q.iy, q.iz, kk);
    const double k2 = kk[0] * kk[0] + kk[1] * kk[1] + kk[2] * kk[2];
    const double k = sqrt(k2);
    const double inv_k2 = (k > 1e-12) ? 1.0 / k2 : 0.0;
    double2 d[L::NFMT];
#pragma unroll
    for (int c = 0; c < L::NFMT; ++c) d[c] = ld2(dk, c * Nk + idx);
    double km[3];
    double2 dm[L::NFMT];
    if (q.proj) {
      const int mx = (p.nx - q.ix) % p.nx;
      const int my = (p.ny - q.iy) % p.ny;
      k_components(p, mx, my, q.iz, km);
#pragma unroll
      for (int c = 0; c < L::NFMT; ++c) dm[c] = ld2(dk, c * Nk + q.midx);
    }
#pragma unroll
    for (int s = 0; s < (MULTI ? kMaxSpecies : 1); ++s) {
      if (s < p.S) {
        const KW w = weight_kernels(k, p.R[s]);
        double2 f = bwd_value<MULTI, TENSOR>(s, p, kk, inv_k2, w, d);
        if (q.proj) {
          const double2 fm = bwd_value<MULTI, TENSOR>(s, p, km, inv_k2, w, dm);
          f.x = 0.5 * (f.x + fm.x);
          f.y = 0.5 * (f.y - fm.y);
        }
        st2(fk, s * Nk + idx, f);
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

// Mixed precision, step 1: per-block sums of each species' density.
__global__ void __launch_bounds__(256) k_species_sums(const double* __restrict__ rho, long long N, int S,
                                                      double* __restrict__ partials) {
  double acc[kMaxSpecies] = {0.0, 0.0, 0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s)
      if (s < S) acc[s] += rho[s * N + i];
  block_reduce_store<kMaxSpecies>(acc, S, partials);
}

// Mixed precision, step 2: delta_rho = rho - mean in FP32; block 0 stores the means.
__global__ void __launch_bounds__(256) k_split_convert(const double* __restrict__ rho, long long N, int S,
                                                       const double* __restrict__ partials, int nblocks,
                                                       float* __restrict__ out, double* __restrict__ mean_out) {
  __shared__ double sm[kMaxSpecies];
  const int warp = threadIdx.x >> 5;
  if (warp < S) {
    const double v = warp_sum_partials(partials, nblocks, S, warp);
    if ((threadIdx.x & 31) == 0) sm[warp] = v / (double)N;
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x < S) mean_out[threadIdx.x] = sm[threadIdx.x];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s)
      if (s < S) out[s * N + i] = (float)(rho[s * N + i] - sm[s]);
}

// ------------------------------------------------------------ pointwise

struct PointwiseArgs {
  const double* rho;      // S*N
  const double* vext;     // S*N or null
  double mu[kMaxSpecies];
  double* force;          // S*N: local terms written here
  double* partials;       // gridDim.x * n_terms
  const double* mf_w;     // M*Nk (k = 0 entries give the mean-field DC weights)
  const double* mean;     // S species means (mixed precision) or null
  double* dbar_out;       // derivative-channel constants (mixed precision) or null
};

// Derivative-channel values at one point from dPhi (the folding of
// hard_sphere.hpp:121,125,131 plus the T_zz trace folding).
template <bool MULTI, bool TENSOR>
__device__ __forceinline__ void fold_derivs(const EvalParams& p, const MeasureDerivs<double>& dm, double* D) {
  using L = Lay<MULTI, TENSOR>;
  const double dzz = TENSOR ? dm.d_t[5] : 0.0;
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
template <bool MULTI, bool TENSOR>
__device__ __forceinline__ void assemble(const EvalParams& p, const double* n, Measures<double>& m) {
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
    for (int c = 0; c < 6; ++c) m.t[c] = 0.0;
  }
}

template <bool MULTI, bool TENSOR, typename RT>
__global__ void __launch_bounds__(256) k_pointwise(EvalParams p, const RT* __restrict__ chan, RT* __restrict__ deriv,
                                                   PointwiseArgs a) {
  using L = Lay<MULTI, TENSOR>;
  constexpr bool SPLIT = sizeof(RT) == sizeof(float);
  constexpr int NT = 4 + kMaxSpecies;
  constexpr int NF = L::NFMT;
  __shared__ double s_off[kMaxChannels];
  __shared__ double s_dbar[NF];
  if (SPLIT) {
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
      if (fmt_phi_dphi<double>(p.model, p.A, p.B, TENSOR, m0, phi0, d0)) {
        fold_derivs<MULTI, TENSOR>(p, d0, D0);
      } else {
#pragma unroll
        for (int c = 0; c < NF; ++c) D0[c] = 0.0;
      }
#pragma unroll
      for (int c = 0; c < NF; ++c) {
        s_dbar[c] = D0[c];
        if (blockIdx.x == 0) a.dbar_out[c] = D0[c];
      }
    }
    __syncthreads();
  }
  const long long N = p.N;
  double acc[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) acc[t] = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
       idx += (long long)gridDim.x * blockDim.x) {
    double n[NF];
#pragma unroll
    for (int c = 0; c < NF; ++c) n[c] = (double)chan[c * N + idx] + (SPLIT ? s_off[c] : 0.0);
    Measures<double> m;
    assemble<MULTI, TENSOR>(p, n, m);
    double phi = 0.0;
    MeasureDerivs<double> dm;
    double D[NF];
    if (fmt_phi_dphi<double>(p.model, p.A, p.B, TENSOR, m, phi, dm)) {
      fold_derivs<MULTI, TENSOR>(p, dm, D);
    } else {
      phi = 0.0;
#pragma unroll
      for (int c = 0; c < NF; ++c) D[c] = 0.0;
    }
    acc[kTermHS] += phi;
#pragma unroll
    for (int c = 0; c < NF; ++c) deriv[c * N + idx] = (RT)(SPLIT ? D[c] - s_dbar[c] : D[c]);
    // ideal gas, external field, mean field (local parts of the force)
    double f[kMaxSpecies];
    double rs[kMaxSpecies];
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
      if (s < p.S) {
        const double r = a.rho[s * N + idx];
        const double v = a.vext ? a.vext[s * N + idx] : 0.0;
        const double lr = log(r < 1e-300 ? 1e-300 : r);
        rs[s] = r;
        acc[kTermId] += r * (lr - 1.0);
        acc[kTermExt] += r * v;
        acc[kTermN0 + s] += r;
        f[s] = (lr - a.mu[s]) * p.dv + v * p.dv;
      }
    }
    for (int q = 0; q < p.M; ++q) {
      const int i = p.mf_i[q], j = p.mf_j[q];
      const int cjx = p.mf_chan_j[q];
      const double cj = (double)chan[cjx * N + idx] + (SPLIT ? s_off[cjx] : 0.0);
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
        const int cix = p.mf_chan_i[q];
        const double ci = (double)chan[cix * N + idx] + (SPLIT ? s_off[cix] : 0.0);
#pragma unroll
        for (int s = 0; s < kMaxSpecies; ++s) {
          if (s == i) f[s] += 0.5 * cj * p.dv;
          if (s == j) f[s] += 0.5 * ci * p.dv;
        }
      }
    }
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s)
      if (s < p.S) a.force[s * N + idx] = f[s];
  }
  block_reduce_store<NT>(acc, p.n_terms, a.partials);
}

// force_s += c2r(F_s) dV (+ the FP64 constant of the split derivative channels)
// (hard_sphere.hpp:250-253)
template <bool MULTI, bool TENSOR, typename RT>
__global__ void __launch_bounds__(256) k_epilogue(EvalParams p, const RT* __restrict__ hs, const double* __restrict__ dbar,
                                                  double* __restrict__ force) {
  using L = Lay<MULTI, TENSOR>;
  constexpr bool SPLIT = sizeof(RT) == sizeof(float);
  __shared__ double s_const[kMaxSpecies];
  if (SPLIT) {
    if (threadIdx.x < p.S) {
      const int s = threadIdx.x;
      double v = 0.0;
#pragma unroll
      for (int c = 0; c < L::NFMT; ++c) v += chan_dc<MULTI, TENSOR>(c, s, p) * dbar[c];
      s_const[s] = v * p.dv;
    }
    __syncthreads();
  }
  const long long N = p.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
      if (s < p.S) {
        double v = force[s * N + i] + (double)hs[s * N + i] * p.dv;
        if (SPLIT) v += s_const[s];
        force[s * N + i] = v;
      }
    }
}

// Deterministic second reduction stage; writes the scalar block
// [F, Omega, F_id, F_ext, F_hs, F_mf, N_0 .. N_{S-1}] (functionals.hpp:72-92).
struct MuArgs {
  double mu[kMaxSpecies];
};

__global__ void k_reduce_final(const double* __restrict__ partials, int nblocks, EvalParams p, MuArgs mu,
                               double* __restrict__ out) {
  __shared__ double sh[4 + kMaxSpecies];
  const int warp = threadIdx.x >> 5;  // one warp per term
  const int n_terms = p.n_terms;
  if (warp < n_terms) {
    const double v = warp_sum_partials(partials, nblocks, n_terms, warp);
    if ((threadIdx.x & 31) == 0) sh[warp] = v;
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
    for (int s = 0; s < p.S; ++s) muN += mu.mu[s] * sh[kTermN0 + s] * dv;
    out[0] = F;
    out[1] = F - muN;
    out[2] = f_id;
    out[3] = f_ext;
    out[4] = f_hs;
    out[5] = f_mf;
    for (int s = 0; s < p.S; ++s) out[6 + s] = sh[kTermN0 + s] * dv;
  }
}

}  // namespace cdft
