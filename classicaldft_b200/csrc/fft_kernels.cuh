// The fused transform path of one evaluation (mixed precision, power-of-two
// grids with a specialisation in fused.cu): the 3-D R2C / C2R are split
// into a plane pass (z and y, one x-plane per CTA, the whole plane in shared
// memory) and a column pass (x, a tile of columns per CTA), and the k-space
// stages ride on the column pass:
//
//   k_plane_fwd<double>  rho - mean -> FP32, R2C z, FFT y          -> P_rho
//   k_col_fwd            FFT x, channels W_c(k) rho_k, IFFT x      -> Q_c
//   k_plane_inv          IFFT y, C2R z                             -> channels (real)
//   k_pointwise_tma      (unchanged)                               -> derivatives
//   k_plane_fwd<float>   R2C z, FFT y of every derivative          -> P_d
//   k_col_bwd            FFT x, F_s = sum_c conj(W_cs) D_c, IFFT x -> P_f
//   k_plane_inv_epi      IFFT y, C2R z, force += hs dV + const, scalars
//
// so every array is read and written once per pass and no k-space array
// makes a round trip through HBM between its transform and its use.  The
// stage formulas are those of eval_kernels.cuh (fwd_value / bwd_value with
// the symmetrised weights, so the C2R input is Hermitian); the transforms
// are fft_core.cuh's.  DIF leaves x-spectra in digit order; the k-space
// products are pointwise, so the column pass multiplies in that order and
// the inverse DIT restores natural order without a permutation.
//
// The grid dimensions are template parameters: every stage length, span and
// item decomposition is a compile-time constant, so the butterfly index
// arithmetic is shifts, masks and constant multiplies.
#pragma once

#include <type_traits>

#include "eval_kernels.cuh"
#include "fft_core.cuh"

namespace cdft {

constexpr int kPlaneThreads = 256;     // plane passes over many sequences
constexpr int kPlaneThreadsWide = 512;  // plane passes with one sequence per plane (rho, force)
constexpr int kColThreads = 256;

template <int I, int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, N>(f);
  }
}

// One stage's butterfly on the sequence at x (element e at x[e * stride]).
template <int M, int ST, bool INV, bool DIT>
__device__ __forceinline__ void stage_item(fft::cpx* x, int stride, int w, const fft::cpx* tw) {
  constexpr int R = fft::stage_radix(M, ST);
  constexpr int L = fft::dif_length(M, ST);
  if constexpr (DIT)
    fft::dit_item_r<R, INV>(x, stride, M, L, w, tw);
  else
    fft::dif_item_r<R, INV>(x, stride, M, L, w, tw);
}

// All stages (DIF in plan order, or DIT in reverse) of NSEQ sequences of
// length M: sequence c starts at base + c * SEQ_STEP, element stride STRIDE.
// Neighbouring threads take neighbouring sequences (or, with ITEM_FAST,
// neighbouring butterflies of one sequence).
template <int M, bool INV, bool DIT, int NT, int NSEQ, int SEQ_STEP, int STRIDE, bool ITEM_FAST>
__device__ __forceinline__ void fft_seqs(fft::cpx* base, const fft::cpx* tw) {
  constexpr int NS = fft::n_stages(M);
  static_for<0, NS>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    constexpr int ST = DIT ? NS - 1 - k : k;
    constexpr int PER = M / fft::stage_radix(M, ST);
    constexpr int ITEMS = NSEQ * PER;
    for (int t = threadIdx.x; t < ITEMS; t += NT) {
      const int c = ITEM_FAST ? t / PER : t % NSEQ;
      const int w = ITEM_FAST ? t % PER : t / NSEQ;
      stage_item<M, ST, INV, DIT>(base + c * SEQ_STEP, STRIDE, w, tw);
    }
    __syncthreads();
  });
}

// All stages along x of `ntiles` column tiles (tile t at buf + t * (M << ltq),
// 2^ltq columns of M rows, row stride 2^ltq).  Powers of two throughout, so
// the item decomposition is shifts and masks.
template <int M, bool INV, bool DIT, int NT>
__device__ __forceinline__ void fft_tiles(fft::cpx* buf, int ntiles, int ltq, const fft::cpx* tw) {
  constexpr int NS = fft::n_stages(M);
  constexpr int LM = fft::ilog2(M);
  const int tq = 1 << ltq;
  static_for<0, NS>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    constexpr int ST = DIT ? NS - 1 - k : k;
    constexpr int LPER = LM - fft::ilog2(fft::stage_radix(M, ST));
    const int lpt = ltq + LPER;  // log2 of the items per tile
    const int items = ntiles << lpt;
    for (int t = threadIdx.x; t < items; t += NT) {
      const int tile = t >> lpt, r = t & ((1 << lpt) - 1);
      const int q = r & (tq - 1), w = r >> ltq;
      stage_item<M, ST, INV, DIT>(buf + ((size_t)tile << (LM + ltq)) + q, tq, w, tw);
    }
    __syncthreads();
  });
}

// ------------------------------------------------------------ plane pass

template <int NY, int NZ, int NT>
struct Plane {
  static constexpr int MZ = NZ / 2, LD = MZ + 1;
  static constexpr size_t kSmem =
      sizeof(fft::cpx) * ((size_t)NY * LD + NY + MZ + NZ) + sizeof(int) * ((size_t)NY + MZ) + 16;
  fft::cpx* P;
  fft::cpx* ty;
  fft::cpx* tz;
  fft::cpx* t2;
  int* slot_y;
  int* slot_z;

  __device__ Plane(unsigned char* base, const FftTables& T) {
    P = reinterpret_cast<fft::cpx*>(base);
    ty = P + (size_t)NY * LD;
    tz = ty + NY;
    t2 = tz + MZ;
    slot_y = reinterpret_cast<int*>(t2 + NZ);
    slot_z = slot_y + NY;
    for (int i = threadIdx.x; i < NY; i += NT) {
      ty[i] = T.ty[i];
      slot_y[i] = fft::dif_slot(NY, i);
    }
    for (int i = threadIdx.x; i < MZ; i += NT) {
      tz[i] = T.tz[i];
      slot_z[i] = fft::dif_slot(MZ, i);
    }
    for (int i = threadIdx.x; i < NZ; i += NT) t2[i] = T.t2[i];
  }

  // y transform of every column kz (DIF: natural in, slot_y order out)
  template <bool INV>
  __device__ __forceinline__ void y_dif() {
    fft_seqs<NY, INV, false, NT, LD, 1, LD, false>(P, ty);
  }
};

// Forward plane pass: R2C along z, FFT along y, store natural order.
// IN = double: rho with the species mean subtracted (the mixed-precision
// split); IN = float: a derivative channel as is.
template <int NY, int NZ, typename IN, int NT>
__global__ void __launch_bounds__(NT, NT == kPlaneThreads ? 3 : 1)
    k_plane_fwd(EvalParams p, const IN* __restrict__ in, int nseq, const double* __restrict__ mean,
                fft::cpx* __restrict__ out, FftTables T) {
  using PL = Plane<NY, NZ, NT>;
  constexpr int MZ = PL::MZ, LD = PL::LD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ix = blockIdx.x, sq = blockIdx.y, b = blockIdx.z;
  PL s(smem_raw, T);
  __syncthreads();
  const IN* src = in + ((long long)b * nseq + sq) * p.N + (long long)ix * NY * NZ;
  const double c = mean ? mean[b * kMaxSpecies + sq] : 0.0;
  // pairs z[n] = x[2n] + i x[2n+1] into DIT input order
  for (int t = threadIdx.x; t < NY * MZ; t += NT) {
    const int iy = t / MZ, n = t % MZ;
    const IN* q = src + (long long)iy * NZ + 2 * n;  // the caller's buffer: scalar loads
    fft::cpx v;
    if constexpr (sizeof(IN) == 8)
      v = {(float)(q[0] - c), (float)(q[1] - c)};
    else
      v = {q[0], q[1]};
    s.P[iy * LD + s.slot_z[n]] = v;
  }
  __syncthreads();
  // z: DIT, slot order in, natural out; neighbouring threads take
  // neighbouring rows (row stride LD is odd: no bank conflicts)
  fft_seqs<MZ, false, true, NT, NY, LD, 1, false>(s.P, s.tz);
  constexpr int PAIRS = MZ / 2 + 1;
  for (int t = threadIdx.x; t < NY * PAIRS; t += NT) {
    const int row = t / PAIRS, k = t % PAIRS;
    fft::r2c_post_item(s.P + row * LD, 1, MZ, k, s.t2);
  }
  __syncthreads();
  s.template y_dif<false>();
  fft::cpx* dst = out + ((long long)b * nseq + sq) * p.Nk + (long long)ix * NY * LD;
  for (int t = threadIdx.x; t < NY * LD; t += NT) {
    const int ky = t / LD, kz = t % LD;
    dst[t] = s.P[s.slot_y[ky] * LD + kz];
  }
}

// Inverse plane pass shared part: load a natural-order plane, IFFT along y
// (DIF), C2R pre-processing and IFFT along z (DIF).  Afterwards sample
// (iy, 2n | 2n+1) is 2 * (Re | Im) of P[slot_y[iy] * LD + slot_z[n]].
template <int NY, int NZ, int NT>
__device__ __forceinline__ void plane_inverse_core(Plane<NY, NZ, NT>& s, const fft::cpx* __restrict__ src) {
  using PL = Plane<NY, NZ, NT>;
  constexpr int MZ = PL::MZ, LD = PL::LD;
  for (int t = threadIdx.x; t < NY * LD; t += NT) s.P[t] = src[t];
  __syncthreads();
  s.template y_dif<true>();
  constexpr int PAIRS = MZ / 2 + 1;
  for (int t = threadIdx.x; t < NY * PAIRS; t += NT) {
    const int row = t / PAIRS, k = t % PAIRS;
    fft::c2r_pre_item(s.P + row * LD, 1, MZ, k, s.t2);
  }
  __syncthreads();
  fft_seqs<MZ, true, false, NT, NY, LD, 1, false>(s.P, s.tz);
}

// Inverse plane pass of the weighted-density channels -> real FP32 channels.
template <int NY, int NZ>
__global__ void __launch_bounds__(kPlaneThreads, 3)
    k_plane_inv(EvalParams p, const fft::cpx* __restrict__ in, int nseq, float* __restrict__ out, FftTables T) {
  constexpr int NT = kPlaneThreads;
  using PL = Plane<NY, NZ, NT>;
  constexpr int MZ = PL::MZ, LD = PL::LD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ix = blockIdx.x, sq = blockIdx.y, b = blockIdx.z;
  PL s(smem_raw, T);
  __syncthreads();
  plane_inverse_core<NY, NZ, NT>(s, in + ((long long)b * nseq + sq) * p.Nk + (long long)ix * NY * LD);
  float* dst = out + ((long long)b * nseq + sq) * p.N + (long long)ix * NY * NZ;  // engine buffer: 8-byte aligned
  for (int t = threadIdx.x; t < NY * MZ; t += NT) {
    const int iy = t / MZ, n = t % MZ;
    const fft::cpx v = s.P[s.slot_y[iy] * LD + s.slot_z[n]];
    *reinterpret_cast<float2*>(dst + (long long)iy * NZ + 2 * n) = make_float2(2.0f * v.x, 2.0f * v.y);
  }
}

// Inverse plane pass of the back-convolved force spectra with the epilogue:
// force_s += hs dV - mu_s dV + (split constant) in FP64.  The CTA of plane
// 0, species 0 of each problem also reduces the pointwise partials into the
// scalar block (the pointwise kernel completed before this launch).
template <int NY, int NZ, bool MULTI, bool TENSOR>
__global__ void __launch_bounds__(kPlaneThreadsWide, 1)
    k_plane_inv_epi(EvalParams p, const fft::cpx* __restrict__ in, const double* __restrict__ dbar,
                    double* __restrict__ force, const __grid_constant__ MuArgs mu, FinalArgs fin, FftTables T) {
  constexpr int NT = kPlaneThreadsWide;
  using PL = Plane<NY, NZ, NT>;
  using L = Lay<MULTI, TENSOR>;
  constexpr int MZ = PL::MZ, LD = PL::LD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ix = blockIdx.x, sp = blockIdx.y, b = blockIdx.z;
  if (ix == 0 && sp == 0 && fin.scalars)
    reduce_final(fin.partials + (long long)b * fin.nblocks * p.n_terms, fin.nblocks, p, mu.mu[b], fin.err,
                 fin.scalars + b * kScalarCount);
  // the force plane is read at the end: start pulling it into L2 now
  {
    const char* fp = reinterpret_cast<const char*>(force + ((long long)b * p.S + sp) * p.N + (long long)ix * NY * NZ);
    for (int off = threadIdx.x * 128; off < NY * NZ * 8; off += NT * 128)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(fp + off));
  }
  PL s(smem_raw, T);
  __shared__ double s_const;
  if (threadIdx.x == 0) {
    double v = 0.0;
    const double* db = dbar + b * kMaxChannels;
#pragma unroll
    for (int c = 0; c < L::NFMT; ++c) v += chan_dc<MULTI, TENSOR>(c, sp, p) * db[c];
    s_const = v * p.dv - mu.mu[b][sp] * p.dv;
  }
  __syncthreads();
  plane_inverse_core<NY, NZ, NT>(s, in + ((long long)b * p.S + sp) * p.Nk + (long long)ix * NY * LD);
  double* dst = force + ((long long)b * p.S + sp) * p.N + (long long)ix * NY * NZ;
  const double dv = p.dv, cst = s_const;
  for (int t = threadIdx.x; t < NY * MZ; t += NT) {
    const int iy = t / MZ, n = t % MZ;
    const fft::cpx v = s.P[s.slot_y[iy] * LD + s.slot_z[n]];
    double* f = dst + (long long)iy * NZ + 2 * n;  // the caller's buffer: 8-byte alignment suffices
    f[0] = f[0] + (double)(2.0f * v.x) * dv + cst;
    f[1] = f[1] + (double)(2.0f * v.y) * dv + cst;
  }
}

// ----------------------------------------------------------- column pass

// Shared memory of a column kernel: the x twiddles and row table, then nbuf
// tiles of nx rows x 2^ltq columns.
__host__ __device__ inline size_t col_smem(int nx, int ltq, int nbuf) {
  return 16 * ((sizeof(fft::cpx) * nx + sizeof(int) * nx + 15) / 16) + sizeof(fft::cpx) * ((size_t)nbuf * nx << ltq);
}

// x transform of `ntiles` tiles (tile t at buf + t * (NX << ltq), row stride 2^ltq).
template <int NX, bool INV, bool DIT>
__device__ __forceinline__ void col_x(fft::cpx* buf, int ntiles, int ltq, const fft::cpx* tx) {
  fft_tiles<NX, INV, DIT, kColThreads>(buf, ntiles, ltq, tx);
}

// Weight table of the column pass, built once per engine (k_build_weights):
// for every half-spectrum index k (natural order), 1/|k|^2 and, per species,
// the |k|-only factors (w3, w2, fv, A, B) of weight_kernels, FP64-computed
// and rounded to FP32 (the precision of the products they multiply).
// Layout: [1 + 5 S][Nk] floats.
__host__ __device__ inline long long weight_table_floats(const EvalParams& p) { return (1 + 5LL * p.S) * p.Nk; }

static __global__ void __launch_bounds__(256) k_build_weights(EvalParams p, float* __restrict__ tab) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < p.Nk;
       idx += (long long)gridDim.x * blockDim.x) {
    const KIndex q = decode_k(p, idx);
    double kk[3], km[3], k, inv_k2;
    k_setup(p, q, kk, km, k, inv_k2);
    tab[idx] = (float)inv_k2;
    for (int s = 0; s < p.S; ++s) {
      const KW w = weight_kernels(k, p.R[s]);
      float* t = tab + (1 + 5LL * s) * p.Nk + idx;
      t[0] = (float)w.w3;
      t[p.Nk] = (float)w.w2;
      t[2 * p.Nk] = (float)w.fv;
      t[3 * p.Nk] = (float)w.A;
      t[4 * p.Nk] = (float)w.B;
    }
  }
}

// kk and the mirror wavevector km of an index in FP32 (k_setup without |k|).
__device__ __forceinline__ void k_vectors(const EvalParams& p, const KIndex& q, float kk[3], float km[3]) {
  double d[3], m[3];
  k_components(p, q.ix, q.iy, q.iz, d);
  if (q.proj) {
    k_components(p, (p.nx - q.ix) % p.nx, (p.ny - q.iy) % p.ny, q.iz, m);
  } else {
    m[0] = d[0];
    m[1] = d[1];
    m[2] = d[2];
  }
  for (int a = 0; a < 3; ++a) {
    kk[a] = (float)d[a];
    km[a] = (float)m[a];
  }
}

__device__ __forceinline__ KWT<float> table_kw(const float* __restrict__ tab, long long Nk, int s, long long idx) {
  const float* t = tab + (1 + 5LL * s) * Nk + idx;
  KWT<float> w;
  w.w3 = t[0];
  w.w2 = t[Nk];
  w.fv = t[2 * Nk];
  w.A = t[3 * Nk];
  w.B = t[4 * Nk];
  return w;
}

__device__ __forceinline__ float2 c2f(fft::cpx v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ fft::cpx f2c(float2 v) { return {v.x, v.y}; }

// The wavevector indices of tile element (row, q): row holds frequency
// kx_of_row[row] after the forward DIF; q is the in-plane index.
__device__ __forceinline__ KIndex col_kindex(const EvalParams& p, int kx, long long q) {
  KIndex ki;
  ki.ix = kx;
  ki.iy = (int)(q / p.nzh);
  ki.iz = (int)(q - (long long)ki.iy * p.nzh);
  ki.proj = (ki.iz == 0) || (((p.nz & 1) == 0) && ki.iz == p.nz / 2);
  return ki;
}

// Column pass of the forward stage: rho_k along x, every weighted-density
// channel (and mean-field convolution) in k-space, inverse x.  Tile: in-plane
// indices q0 .. q0 + TQ - 1 of all NX planes.
template <int NX, bool MULTI, bool TENSOR>
__global__ void __launch_bounds__(kColThreads, 3)
    k_col_fwd(EvalParams p, const fft::cpx* __restrict__ prho, const double* __restrict__ mf_w,
              const float* __restrict__ wtab, fft::cpx* __restrict__ q_out, int ltq, FftTables T) {
  using Ly = Lay<MULTI, TENSOR>;
  constexpr int LNX = fft::ilog2(NX);
  const int TQ = 1 << ltq, LT = LNX + ltq, TILE = 1 << LT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int S = p.S, C = p.n_chan;
  const long long plane = (long long)p.ny * p.nzh;
  const int b = blockIdx.y;
  const long long q0 = (long long)blockIdx.x * TQ;
  fft::cpx* tx = reinterpret_cast<fft::cpx*>(smem_raw);
  int* kx_of_row = reinterpret_cast<int*>(tx + NX);
  fft::cpx* R = reinterpret_cast<fft::cpx*>(smem_raw + 16 * ((sizeof(fft::cpx) * NX + sizeof(int) * NX + 15) / 16));
  fft::cpx* Ch = R + (size_t)S * TILE;
  for (int i = threadIdx.x; i < NX; i += kColThreads) {
    tx[i] = T.tx[i];
    kx_of_row[i] = fft::dif_order(NX, i);
  }
  for (int t = threadIdx.x; t < S * TILE; t += kColThreads) {
    const int sp = t >> LT, e = t & (TILE - 1), ix = e >> ltq, qq = e & (TQ - 1);
    const long long q = q0 + qq;
    R[t] = (q < plane) ? prho[((long long)b * S + sp) * p.Nk + ix * plane + q] : fft::cpx{0.0f, 0.0f};
  }
  __syncthreads();
  col_x<NX, false, false>(R, S, ltq, tx);
  // k-space products, one element per thread iteration (FP64 weights)
  for (int e = threadIdx.x; e < TILE; e += kColThreads) {
    const int row = e >> ltq, qq = e & (TQ - 1);
    const long long q = q0 + qq;
    if (q >= plane) {
      for (int c = 0; c < C; ++c) Ch[(size_t)c * TILE + e] = fft::cpx{0.0f, 0.0f};
      continue;
    }
    const KIndex ki = col_kindex(p, kx_of_row[row], q);
    const long long kidx = (long long)ki.ix * plane + q;
    float kk[3], km[3];
    k_vectors(p, ki, kk, km);
    const float inv_k2 = wtab[kidx];
    KWT<float> kw[kMaxSpecies];
    float2 r[kMaxSpecies];
#pragma unroll
    for (int sp = 0; sp < kMaxSpecies; ++sp) {
      if (sp < S) {
        kw[sp] = table_kw(wtab, p.Nk, sp, kidx);
        r[sp] = c2f(R[(size_t)sp * TILE + e]);
      }
    }
#pragma unroll
    for (int c = 0; c < Ly::NFMT; ++c)
      Ch[(size_t)c * TILE + e] = f2c(fwd_value<MULTI, TENSOR, float, float2>(c, p, kk, km, ki.proj, inv_k2, kw, r));
    // mean-field convolutions (the weight is real and even); rho_k from the
    // tile, not the register array, so no dynamic register index
    for (int m = 0; m < p.M; ++m) {
      const float w = (float)mf_w[m * p.Nk + kidx];
      const float2 rv = c2f(R[(size_t)p.mf_j[m] * TILE + e]);
      Ch[(size_t)p.mf_chan_j[m] * TILE + e] = fft::cpx{w * rv.x, w * rv.y};
      if (p.mf_chan_i[m] >= 0) {
        const float2 ri = c2f(R[(size_t)p.mf_i[m] * TILE + e]);
        Ch[(size_t)p.mf_chan_i[m] * TILE + e] = fft::cpx{w * ri.x, w * ri.y};
      }
    }
  }
  __syncthreads();
  col_x<NX, true, true>(Ch, C, ltq, tx);
  for (int t = threadIdx.x; t < C * TILE; t += kColThreads) {
    const int c = t >> LT, e = t & (TILE - 1), ix = e >> ltq, qq = e & (TQ - 1);
    const long long q = q0 + qq;
    if (q < plane) q_out[((long long)b * C + c) * p.Nk + ix * plane + q] = Ch[t];
  }
}

// Column pass of the backward stage: every derivative channel along x, the
// back-convolution F_s = sum_c conj(W'_cs) D_c, inverse x of F_s.
template <int NX, bool MULTI, bool TENSOR>
__global__ void __launch_bounds__(kColThreads, 3)
    k_col_bwd(EvalParams p, const fft::cpx* __restrict__ pd, const float* __restrict__ wtab, fft::cpx* __restrict__ pf,
              int ltq, FftTables T) {
  using Ly = Lay<MULTI, TENSOR>;
  constexpr int NF = Ly::NFMT;
  constexpr int LNX = fft::ilog2(NX);
  const int TQ = 1 << ltq, LT = LNX + ltq, TILE = 1 << LT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int S = p.S;
  const long long plane = (long long)p.ny * p.nzh;
  const int b = blockIdx.y;
  const long long q0 = (long long)blockIdx.x * TQ;
  fft::cpx* tx = reinterpret_cast<fft::cpx*>(smem_raw);
  int* kx_of_row = reinterpret_cast<int*>(tx + NX);
  fft::cpx* Dt = reinterpret_cast<fft::cpx*>(smem_raw + 16 * ((sizeof(fft::cpx) * NX + sizeof(int) * NX + 15) / 16));
  for (int i = threadIdx.x; i < NX; i += kColThreads) {
    tx[i] = T.tx[i];
    kx_of_row[i] = fft::dif_order(NX, i);
  }
  for (int t = threadIdx.x; t < NF * TILE; t += kColThreads) {
    const int c = t >> LT, e = t & (TILE - 1), ix = e >> ltq, qq = e & (TQ - 1);
    const long long q = q0 + qq;
    Dt[t] = (q < plane) ? pd[((long long)b * NF + c) * p.Nk + ix * plane + q] : fft::cpx{0.0f, 0.0f};
  }
  __syncthreads();
  col_x<NX, false, false>(Dt, NF, ltq, tx);
  // species force spectra overwrite tiles 0 .. S-1 (each element is read in
  // full before it is written, and elements are independent)
  for (int e = threadIdx.x; e < TILE; e += kColThreads) {
    const int row = e >> ltq, qq = e & (TQ - 1);
    const long long q = q0 + qq;
    if (q >= plane) continue;
    const KIndex ki = col_kindex(p, kx_of_row[row], q);
    const long long kidx = (long long)ki.ix * plane + q;
    float kk[3], km[3];
    k_vectors(p, ki, kk, km);
    const float inv_k2 = wtab[kidx];
    float2 d[NF];
#pragma unroll
    for (int c = 0; c < NF; ++c) d[c] = c2f(Dt[(size_t)c * TILE + e]);
#pragma unroll
    for (int sp = 0; sp < (MULTI ? kMaxSpecies : 1); ++sp) {
      if (sp < S) {
        const KWT<float> w = table_kw(wtab, p.Nk, sp, kidx);
        Dt[(size_t)sp * TILE + e] = f2c(bwd_value<MULTI, TENSOR, float, float2>(sp, p, kk, km, ki.proj, inv_k2, w, d));
      }
    }
  }
  __syncthreads();
  col_x<NX, true, true>(Dt, S, ltq, tx);
  for (int t = threadIdx.x; t < S * TILE; t += kColThreads) {
    const int sp = t >> LT, e = t & (TILE - 1), ix = e >> ltq, qq = e & (TQ - 1);
    const long long q = q0 + qq;
    if (q < plane) pf[((long long)b * S + sp) * p.Nk + ix * plane + q] = Dt[t];
  }
}

}  // namespace cdft
