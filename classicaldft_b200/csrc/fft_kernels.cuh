// The fused transform path of one evaluation (mixed precision, power-of-two
// grids whose (y, z) planes fit in shared memory): the 3-D R2C / C2R are
// split into a plane pass (z and y, one x-plane per CTA, the whole plane in
// shared memory) and a column pass (x, a tile of columns per CTA), and the
// k-space stages ride on the column pass:
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
#pragma once

#include "eval_kernels.cuh"
#include "fft_core.cuh"

namespace cdft {

constexpr int kPlaneThreads = 512;
constexpr int kColThreads = 256;

// Shared-memory layout of a plane kernel: the plane (ny rows of nz/2 + 1
// complex), twiddles, then the digit-order slot tables.
struct PlaneSmem {
  fft::cpx* P;
  fft::cpx* ty;
  fft::cpx* tz;
  fft::cpx* t2;
  int* slot_y;
  int* slot_z;
};

__host__ __device__ inline size_t plane_smem_bytes(int ny, int nz) {
  const int Mz = nz / 2;
  return sizeof(fft::cpx) * ((size_t)ny + Mz + nz + (size_t)ny * (Mz + 1)) + sizeof(int) * ((size_t)ny + Mz) + 16;
}

__device__ inline PlaneSmem plane_smem(unsigned char* base, int ny, int nz) {
  const int Mz = nz / 2;
  PlaneSmem s;
  s.P = reinterpret_cast<fft::cpx*>(base);
  s.ty = s.P + (size_t)ny * (Mz + 1);
  s.tz = s.ty + ny;
  s.t2 = s.tz + Mz;
  s.slot_y = reinterpret_cast<int*>(s.t2 + nz);
  s.slot_z = s.slot_y + ny;
  return s;
}

__device__ inline void plane_tables(const PlaneSmem& s, const FftTables& T, int ny, int nz) {
  const int Mz = nz / 2;
  for (int i = threadIdx.x; i < ny; i += blockDim.x) {
    s.ty[i] = T.ty[i];
    s.slot_y[i] = fft::dif_slot(ny, i);
  }
  for (int i = threadIdx.x; i < Mz; i += blockDim.x) {
    s.tz[i] = T.tz[i];
    s.slot_z[i] = fft::dif_slot(Mz, i);
  }
  for (int i = threadIdx.x; i < nz; i += blockDim.x) s.t2[i] = T.t2[i];
}

// All stages of the y transform of the plane (columns of ld complex rows):
// DIF, natural in, digit order (slot_y) out.
template <bool INV>
__device__ inline void plane_y_dif(const PlaneSmem& s, int ny, int ld) {
  const int ns = fft::n_stages(ny);
  for (int st = 0; st < ns; ++st) {
    const int r = fft::stage_radix(ny, st), L = fft::dif_length(ny, st);
    const int items = ld * (ny / r);
    for (int t = threadIdx.x; t < items; t += blockDim.x) {
      const int col = t % ld, w = t / ld;
      fft::dif_item<INV>(s.P + col, ld, ny, L, r, w, s.ty);
    }
    __syncthreads();
  }
}

// Forward plane pass: R2C along z, FFT along y, store natural order.
// IN = double: rho with the species mean subtracted (the mixed-precision
// split); IN = float: a derivative channel as is.
template <typename IN>
__global__ void __launch_bounds__(kPlaneThreads, 2)
    k_plane_fwd(EvalParams p, const IN* __restrict__ in, int nseq, const double* __restrict__ mean,
                fft::cpx* __restrict__ out, FftTables T) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ny = p.ny, nz = p.nz, Mz = nz / 2, ld = Mz + 1;
  const int ix = blockIdx.x, sq = blockIdx.y, b = blockIdx.z;
  const PlaneSmem s = plane_smem(smem_raw, ny, nz);
  plane_tables(s, T, ny, nz);
  __syncthreads();
  const IN* src = in + ((long long)b * nseq + sq) * p.N + (long long)ix * ny * nz;
  const double c = mean ? mean[b * kMaxSpecies + sq] : 0.0;
  // pairs z[n] = x[2n] + i x[2n+1] into DIT input order
  for (int t = threadIdx.x; t < ny * Mz; t += blockDim.x) {
    const int iy = t / Mz, n = t - iy * Mz;
    const IN* q = src + (long long)iy * nz + 2 * n;  // the caller's buffer: scalar loads
    fft::cpx v;
    if constexpr (sizeof(IN) == 8)
      v = {(float)(q[0] - c), (float)(q[1] - c)};
    else
      v = {q[0], q[1]};
    s.P[iy * ld + s.slot_z[n]] = v;
  }
  __syncthreads();
  // z: DIT (slot order in, natural out), stages in reverse
  const int nsz = fft::n_stages(Mz);
  for (int st = nsz - 1; st >= 0; --st) {
    const int r = fft::stage_radix(Mz, st), L = fft::dif_length(Mz, st);
    const int per = Mz / r;
    for (int t = threadIdx.x; t < ny * per; t += blockDim.x) {
      const int row = t / per, w = t - row * per;
      fft::dit_item<false>(s.P + row * ld, 1, Mz, L, r, w, s.tz);
    }
    __syncthreads();
  }
  const int pairs = Mz / 2 + 1;
  for (int t = threadIdx.x; t < ny * pairs; t += blockDim.x) {
    const int row = t / pairs, k = t - row * pairs;
    fft::r2c_post_item(s.P + row * ld, 1, Mz, k, s.t2);
  }
  __syncthreads();
  plane_y_dif<false>(s, ny, ld);
  fft::cpx* dst = out + ((long long)b * nseq + sq) * p.Nk + (long long)ix * ny * ld;
  for (int t = threadIdx.x; t < ny * ld; t += blockDim.x) {
    const int ky = t / ld, kz = t - ky * ld;
    dst[t] = s.P[s.slot_y[ky] * ld + kz];
  }
}

// Inverse plane pass shared part: load a natural-order plane, IFFT along y
// (DIF), C2R pre-processing and IFFT along z (DIF).  Afterwards sample
// (iy, 2n | 2n+1) is 2 * (Re | Im) of P[slot_y[iy] * ld + slot_z[n]].
__device__ inline void plane_inverse_core(const PlaneSmem& s, const fft::cpx* __restrict__ src, int ny, int nz) {
  const int Mz = nz / 2, ld = Mz + 1;
  for (int t = threadIdx.x; t < ny * ld; t += blockDim.x) s.P[t] = src[t];
  __syncthreads();
  plane_y_dif<true>(s, ny, ld);
  const int pairs = Mz / 2 + 1;
  for (int t = threadIdx.x; t < ny * pairs; t += blockDim.x) {
    const int row = t / pairs, k = t - row * pairs;
    fft::c2r_pre_item(s.P + row * ld, 1, Mz, k, s.t2);
  }
  __syncthreads();
  const int nsz = fft::n_stages(Mz);
  for (int st = 0; st < nsz; ++st) {
    const int r = fft::stage_radix(Mz, st), L = fft::dif_length(Mz, st);
    const int per = Mz / r;
    for (int t = threadIdx.x; t < ny * per; t += blockDim.x) {
      const int row = t / per, w = t - row * per;
      fft::dif_item<true>(s.P + row * ld, 1, Mz, L, r, w, s.tz);
    }
    __syncthreads();
  }
}

// Inverse plane pass of the weighted-density channels -> real FP32 channels.
__global__ void __launch_bounds__(kPlaneThreads, 2)
    k_plane_inv(EvalParams p, const fft::cpx* __restrict__ in, int nseq, float* __restrict__ out, FftTables T) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ny = p.ny, nz = p.nz, Mz = nz / 2, ld = Mz + 1;
  const int ix = blockIdx.x, sq = blockIdx.y, b = blockIdx.z;
  const PlaneSmem s = plane_smem(smem_raw, ny, nz);
  plane_tables(s, T, ny, nz);
  __syncthreads();
  plane_inverse_core(s, in + ((long long)b * nseq + sq) * p.Nk + (long long)ix * ny * ld, ny, nz);
  float* dst = out + ((long long)b * nseq + sq) * p.N + (long long)ix * ny * nz;  // engine buffer: 8-byte aligned
  for (int t = threadIdx.x; t < ny * Mz; t += blockDim.x) {
    const int iy = t / Mz, n = t - iy * Mz;
    const fft::cpx v = s.P[s.slot_y[iy] * ld + s.slot_z[n]];
    *reinterpret_cast<float2*>(dst + (long long)iy * nz + 2 * n) = make_float2(2.0f * v.x, 2.0f * v.y);
  }
}

// Inverse plane pass of the back-convolved force spectra with the epilogue:
// force_s += hs dV - mu_s dV + (split constant) in FP64.  The CTA of plane
// 0, species 0 of each problem also reduces the pointwise partials into the
// scalar block (the pointwise kernel completed before this launch).
template <bool MULTI, bool TENSOR>
__global__ void __launch_bounds__(kPlaneThreads, 2)
    k_plane_inv_epi(EvalParams p, const fft::cpx* __restrict__ in, const double* __restrict__ dbar,
                    double* __restrict__ force, const __grid_constant__ MuArgs mu, FinalArgs fin, FftTables T) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using L = Lay<MULTI, TENSOR>;
  const int ny = p.ny, nz = p.nz, Mz = nz / 2, ld = Mz + 1;
  const int ix = blockIdx.x, sp = blockIdx.y, b = blockIdx.z;
  if (ix == 0 && sp == 0 && fin.scalars)
    reduce_final(fin.partials + (long long)b * fin.nblocks * p.n_terms, fin.nblocks, p, mu.mu[b], fin.err,
                 fin.scalars + b * kScalarCount);
  const PlaneSmem s = plane_smem(smem_raw, ny, nz);
  plane_tables(s, T, ny, nz);
  __shared__ double s_const;
  if (threadIdx.x == 0) {
    double v = 0.0;
    const double* db = dbar + b * kMaxChannels;
#pragma unroll
    for (int c = 0; c < L::NFMT; ++c) v += chan_dc<MULTI, TENSOR>(c, sp, p) * db[c];
    s_const = v * p.dv - mu.mu[b][sp] * p.dv;
  }
  __syncthreads();
  plane_inverse_core(s, in + ((long long)b * p.S + sp) * p.Nk + (long long)ix * ny * ld, ny, nz);
  double* dst = force + ((long long)b * p.S + sp) * p.N + (long long)ix * ny * nz;
  const double dv = p.dv, cst = s_const;
  for (int t = threadIdx.x; t < ny * Mz; t += blockDim.x) {
    const int iy = t / Mz, n = t - iy * Mz;
    const fft::cpx v = s.P[s.slot_y[iy] * ld + s.slot_z[n]];
    double* f = dst + (long long)iy * nz + 2 * n;  // the caller's buffer: 8-byte alignment suffices
    f[0] = f[0] + (double)(2.0f * v.x) * dv + cst;
    f[1] = f[1] + (double)(2.0f * v.y) * dv + cst;
  }
}

// ---------------------------------------------------------- column pass

// Shared-memory bytes of a column kernel: the x twiddles, then nbuf tiles of
// nx rows x tq columns.
__host__ __device__ inline size_t col_smem_bytes(int nx, int tq, int nbuf) {
  return sizeof(fft::cpx) * ((size_t)nx + (size_t)nbuf * nx * tq) + 16;
}

// DIF (forward) or DIT (inverse) along x of `ncols` tile columns (tile t,
// column q of tile buffer at buf + t * nx * tq + q, row stride tq).
template <bool INV, bool DIT>
__device__ inline void col_x_transform(fft::cpx* buf, int nx, int tq, int ncols, const fft::cpx* tx) {
  const int ns = fft::n_stages(nx);
  for (int k = 0; k < ns; ++k) {
    const int st = DIT ? ns - 1 - k : k;
    const int r = fft::stage_radix(nx, st), L = fft::dif_length(nx, st);
    const int per = nx / r;
    for (int t = threadIdx.x; t < ncols * per; t += blockDim.x) {
      const int col = t % ncols, w = t / ncols;
      const int tile = col / tq, q = col - tile * tq;
      fft::cpx* x = buf + (size_t)tile * nx * tq + q;
      if (DIT)
        fft::dit_item<INV>(x, tq, nx, L, r, w, tx);
      else
        fft::dif_item<INV>(x, tq, nx, L, r, w, tx);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double2 c2d(fft::cpx v) { return make_double2((double)v.x, (double)v.y); }
__device__ __forceinline__ fft::cpx d2c(double2 v) { return {(float)v.x, (float)v.y}; }

// The wavevector indices of tile element (row, q): row holds frequency
// dif_order(nx, row) after the forward DIF; q is the in-plane index.
__device__ __forceinline__ KIndex col_kindex(const EvalParams& p, int row, long long q) {
  KIndex ki;
  ki.ix = fft::dif_order(p.nx, row);
  ki.iy = (int)(q / p.nzh);
  ki.iz = (int)(q - (long long)ki.iy * p.nzh);
  ki.proj = (ki.iz == 0) || (((p.nz & 1) == 0) && ki.iz == p.nz / 2);
  return ki;
}

// Column pass of the forward stage: rho_k along x, every weighted-density
// channel (and mean-field convolution) in k-space, inverse x.  Tile: in-plane
// indices q0 .. q0 + tq - 1 of all nx planes.
template <bool MULTI, bool TENSOR>
__global__ void __launch_bounds__(kColThreads, 2)
    k_col_fwd(EvalParams p, const fft::cpx* __restrict__ prho, const double* __restrict__ mf_w,
              fft::cpx* __restrict__ q_out, int tq, FftTables T) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using Ly = Lay<MULTI, TENSOR>;
  const int nx = p.nx, S = p.S, C = p.n_chan;
  const long long plane = (long long)p.ny * p.nzh;
  const int b = blockIdx.y;
  const long long q0 = (long long)blockIdx.x * tq;
  fft::cpx* tx = reinterpret_cast<fft::cpx*>(smem_raw);
  fft::cpx* R = tx + nx;                   // S tiles
  fft::cpx* Ch = R + (size_t)S * nx * tq;  // C tiles
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tx[i] = T.tx[i];
  const int tile = nx * tq;
  for (int t = threadIdx.x; t < S * tile; t += blockDim.x) {
    const int sp = t / tile, e = t - sp * tile, ix = e / tq, qq = e - ix * tq;
    const long long q = q0 + qq;
    R[t] = (q < plane) ? prho[((long long)b * S + sp) * p.Nk + ix * plane + q] : fft::cpx{0.0f, 0.0f};
  }
  __syncthreads();
  col_x_transform<false, false>(R, nx, tq, S * tq, tx);
  // k-space products, one element per thread iteration (FP64 weights)
  for (int e = threadIdx.x; e < tile; e += blockDim.x) {
    const int row = e / tq, qq = e - row * tq;
    const long long q = q0 + qq;
    if (q >= plane) {
      for (int c = 0; c < C; ++c) Ch[(size_t)c * tile + e] = fft::cpx{0.0f, 0.0f};
      continue;
    }
    const KIndex ki = col_kindex(p, row, q);
    double kk[3], km[3], k, inv_k2;
    k_setup(p, ki, kk, km, k, inv_k2);
    KW kw[kMaxSpecies];
    double2 r[kMaxSpecies];
#pragma unroll
    for (int sp = 0; sp < kMaxSpecies; ++sp) {
      if (sp < S) {
        kw[sp] = weight_kernels(k, p.R[sp]);
        r[sp] = c2d(R[(size_t)sp * tile + e]);
      }
    }
#pragma unroll
    for (int c = 0; c < Ly::NFMT; ++c)
      Ch[(size_t)c * tile + e] = d2c(fwd_value<MULTI, TENSOR>(c, p, kk, km, ki.proj, inv_k2, kw, r));
    // mean-field convolutions (the weight is real and even); rho_k from the
    // tile, not the register array, so no dynamic register index
    const long long kidx = (long long)ki.ix * plane + q;
    for (int m = 0; m < p.M; ++m) {
      const double w = mf_w[m * p.Nk + kidx];
      const double2 rv = c2d(R[(size_t)p.mf_j[m] * tile + e]);
      Ch[(size_t)p.mf_chan_j[m] * tile + e] = d2c(make_double2(w * rv.x, w * rv.y));
      if (p.mf_chan_i[m] >= 0) {
        const double2 ri = c2d(R[(size_t)p.mf_i[m] * tile + e]);
        Ch[(size_t)p.mf_chan_i[m] * tile + e] = d2c(make_double2(w * ri.x, w * ri.y));
      }
    }
  }
  __syncthreads();
  col_x_transform<true, true>(Ch, nx, tq, C * tq, tx);
  for (int t = threadIdx.x; t < C * tile; t += blockDim.x) {
    const int c = t / tile, e = t - c * tile, ix = e / tq, qq = e - ix * tq;
    const long long q = q0 + qq;
    if (q < plane) q_out[((long long)b * C + c) * p.Nk + ix * plane + q] = Ch[t];
  }
}

// Column pass of the backward stage: every derivative channel along x, the
// back-convolution F_s = sum_c conj(W'_cs) D_c, inverse x of F_s.
template <bool MULTI, bool TENSOR>
__global__ void __launch_bounds__(kColThreads, 2)
    k_col_bwd(EvalParams p, const fft::cpx* __restrict__ pd, fft::cpx* __restrict__ pf, int tq, FftTables T) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using Ly = Lay<MULTI, TENSOR>;
  constexpr int NF = Ly::NFMT;
  const int nx = p.nx, S = p.S;
  const long long plane = (long long)p.ny * p.nzh;
  const int b = blockIdx.y;
  const long long q0 = (long long)blockIdx.x * tq;
  fft::cpx* tx = reinterpret_cast<fft::cpx*>(smem_raw);
  fft::cpx* Dt = tx + nx;  // NF tiles; species force spectra overwrite tiles 0 .. S-1
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tx[i] = T.tx[i];
  const int tile = nx * tq;
  for (int t = threadIdx.x; t < NF * tile; t += blockDim.x) {
    const int c = t / tile, e = t - c * tile, ix = e / tq, qq = e - ix * tq;
    const long long q = q0 + qq;
    Dt[t] = (q < plane) ? pd[((long long)b * NF + c) * p.Nk + ix * plane + q] : fft::cpx{0.0f, 0.0f};
  }
  __syncthreads();
  col_x_transform<false, false>(Dt, nx, tq, NF * tq, tx);
  for (int e = threadIdx.x; e < tile; e += blockDim.x) {
    const int row = e / tq, qq = e - row * tq;
    const long long q = q0 + qq;
    if (q >= plane) continue;
    const KIndex ki = col_kindex(p, row, q);
    double kk[3], km[3], k, inv_k2;
    k_setup(p, ki, kk, km, k, inv_k2);
    double2 d[NF];
#pragma unroll
    for (int c = 0; c < NF; ++c) d[c] = c2d(Dt[(size_t)c * tile + e]);
#pragma unroll
    for (int sp = 0; sp < (MULTI ? kMaxSpecies : 1); ++sp) {
      if (sp < S) {
        const KW w = weight_kernels(k, p.R[sp]);
        Dt[(size_t)sp * tile + e] = d2c(bwd_value<MULTI, TENSOR>(sp, p, kk, km, ki.proj, inv_k2, w, d));
      }
    }
  }
  __syncthreads();
  col_x_transform<true, true>(Dt, nx, tq, S * tq, tx);
  for (int t = threadIdx.x; t < S * tile; t += blockDim.x) {
    const int sp = t / tile, e = t - sp * tile, ix = e / tq, qq = e - ix * tq;
    const long long q = q0 + qq;
    if (q < plane) pf[((long long)b * S + sp) * p.Nk + ix * plane + q] = Dt[t];
  }
}

}  // namespace cdft
