// Kernels of the fused transform path on register-resident transforms
// (fft_reg.cuh).  A length-N transform is two in-register DFTs (A and B
// points) with one shared-memory exchange between them; a plane pass is a
// y transform and a z transform (three exchanges, with the half-complex
// steps on the y-spectrum), a column pass one x transform per
// array.  The passes and their arrays are those of the stage-by-stage
// kernels they replace:
//
//   k_rplane_fwd<double>  R2C z, FFT y of rho - mean          -> P_rho
//   k_rcol_fwd            FFT x, channels W_c(k) rho_k, IFFT x -> Q_c
//   k_rplane_inv          IFFT y, C2R z                        -> channels (real)
//   (pointwise)
//   k_rplane_fwd<float>   R2C z, FFT y of every derivative     -> P_d
//   k_rcol_bwd            FFT x, F_s = sum_c conj(W_cs) D_c, IFFT x -> P_f
//   k_rplane_inv<EPI>     IFFT y, C2R z, force += hs dV + const, scalars
//
// Every task loop maps consecutive threads to consecutive z (plane) or
// in-plane column (column pass) indices, so global accesses are contiguous
// and shared-memory accesses fall in distinct banks; values a task needs
// after a barrier that also frees the buffer are held in registers.
#pragma once

#include <type_traits>

#include "eval_kernels.cuh"
#include "fft_reg.cuh"

namespace cdft {
namespace rk {

using fft::cpx;

template <int I, int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, N>(f);
  }
}

// Smallest v >= x with v = 8 (mod 16): a row stride that puts rows y and
// y + 1 of a half-warp's 64-bit accesses in different bank halves.
__host__ __device__ constexpr int pad8(int x) { return x + ((8 - x % 16) + 16) % 16; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// ------------------------------------------------------------ plane pass

template <int NY, int NZ>
struct RPlane {
  static constexpr int M = NZ / 2, LD = M + 1;
  using SY = fft::Split<NY>;
  using SZ = fft::Split<M>;
  static constexpr int AY = SY::A, BY = SY::B, AZ = SZ::A, BZ = SZ::B;
  static constexpr int EY = M;               // y exchange: [n2][k1][kz]
  static constexpr int ER = pad8(M);         // rows: [y][kz]
  static constexpr int EZS = AZ + 1;         // z exchange: [y][n2][k1], n2 stride
  static constexpr int EZ = pad8(BZ * EZS);  // z exchange row stride
  static constexpr int BUF = cmax(NY * EY, cmax(NY * ER, NY * EZ));
  static constexpr int NT = NY * M >= 8192 ? 512 : (NY * M >= 2048 ? 256 : 128);
  // the passes with one sequence per plane (rho in, force out) launch one
  // CTA per x plane only: twice the threads per CTA
  static constexpr int NT_WIDE = NT * 2;
  static constexpr size_t kSmem = sizeof(cpx) * ((size_t)BUF + NY + M + NZ);
  // tasks of each phase and the tasks a thread holds across a barrier
  static constexpr int T_Y_SPEC = M * AY, T_Y_NAT = M * BY, T_Z_SPEC = NY * AZ, T_Z_NAT = NY * BZ;
};

template <int NY, int NZ, int NT>
__device__ __forceinline__ void plane_tables(cpx* ty, cpx* tz, cpx* t2, const FftTables& T) {
  for (int i = threadIdx.x; i < NY; i += NT) ty[i] = T.ty[i];
  for (int i = threadIdx.x; i < NZ / 2; i += NT) tz[i] = T.tz[i];
  for (int i = threadIdx.x; i < NZ; i += NT) t2[i] = T.t2[i];
}

// One bulk copy (TMA, no multicast) of `bytes` (a multiple of 16, both
// addresses 16-byte aligned) from global memory into shared dst, waited for
// by every thread with a bound.  False, with *err set, when the wait gave
// up: the block then waits once more (bounded) so a late copy lands before
// it exits, and returns without using the data.
__device__ __forceinline__ bool bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar, int* err) {
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(bar, bytes);
    bulk_copy_g2s(dst, src, bytes, bar);
  }
  const bool ok = mbar_wait_bounded(bar, 0, kWaitLimit);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0 && err) atomicExch(err, 1);
    mbar_wait_bounded(bar, 0, kWaitLimit);
    return false;
  }
  return true;
}

// Forward plane pass of one real NY x NZ plane into its half spectrum
// (NY x (NZ/2 + 1), natural order).  IN = float: a derivative channel.
// IN = double: rho, split for mixed precision around the plane's own mean
// m_x (FP64, written to pmean[(b S + s) nx + ix]): the plane transformed is
// rho - m_x in FP32, and the column pass restores the plane means' profile
// around the species mean (rk_dc_column).
template <int NY, int NZ, typename IN, int NT = RPlane<NY, NZ>::NT>
__global__ void __launch_bounds__(NT)
    k_rplane_fwd(EvalParams p, const IN* __restrict__ in, int nseq, double* __restrict__ pmean,
                 cpx* __restrict__ out, int* err, int ix0, FftTables T) {
  pdl_trigger();
  pdl_wait();
  using P = RPlane<NY, NZ>;
  constexpr int M = P::M, LD = P::LD, AY = P::AY, BY = P::BY, AZ = P::AZ, BZ = P::BZ;
  constexpr int EY = P::EY, ER = P::ER, EZS = P::EZS, EZ = P::EZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx* E = reinterpret_cast<cpx*>(smem_raw);
  cpx* ty = E + P::BUF;
  cpx* tz = ty + NY;
  cpx* t2 = tz + M;
  const int ix = ix0 + blockIdx.x, sq = blockIdx.y, b = blockIdx.z;  // planes ix0 ..
  plane_tables<NY, NZ, NT>(ty, tz, t2, T);
  __syncthreads();
  const IN* src = in + ((long long)b * nseq + sq) * p.N + (long long)ix * NY * NZ;
  if constexpr (sizeof(IN) == 8) {
    // rho (FP64): one read of the plane into registers, its mean (a
    // fixed-order block sum, recorded for the column pass), rho - mean in
    // FP32 into shared memory as the real plane (pairs E[y * M + n])
    // each thread takes pairs of consecutive samples (PER even): one 16-byte
    // load each where rho is 16-byte aligned, two 8-byte loads otherwise
    // (the same samples and summation order either way)
    constexpr int PER = NY * NZ / NT;
    static_assert(PER * NT == NY * NZ, "plane samples per thread");
    constexpr bool PAIRS = PER % 2 == 0;
    double v[PER];
    double sum = 0.0;
    if constexpr (PAIRS) {
      if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
        const double2* src2 = reinterpret_cast<const double2*>(src);
#pragma unroll
        for (int j = 0; j < PER / 2; ++j) {
          const double2 d = src2[threadIdx.x + j * NT];
          v[2 * j] = d.x;
          v[2 * j + 1] = d.y;
        }
      } else {
#pragma unroll
        for (int j = 0; j < PER / 2; ++j) {
          v[2 * j] = src[2 * (threadIdx.x + j * NT)];
          v[2 * j + 1] = src[2 * (threadIdx.x + j * NT) + 1];
        }
      }
#pragma unroll
      for (int j = 0; j < PER / 2; ++j) sum += v[2 * j] + v[2 * j + 1];
    } else {
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        v[j] = src[threadIdx.x + j * NT];
        sum += v[j];
      }
    }
    __shared__ double s_warp[NT / 32];
    __shared__ double s_mean;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
      for (int w = 0; w < NT / 32; ++w) m += s_warp[w];
      m /= (double)(NY * NZ);
      s_mean = m;
      pmean[((long long)b * nseq + sq) * p.nx + ix] = m;
    }
    __syncthreads();
    const double c = s_mean;
    if constexpr (PAIRS) {
      float2* Ef2 = reinterpret_cast<float2*>(E);
#pragma unroll
      for (int j = 0; j < PER / 2; ++j)
        Ef2[threadIdx.x + j * NT] = make_float2((float)(v[2 * j] - c), (float)(v[2 * j + 1] - c));
    } else {
      float* Ef = reinterpret_cast<float*>(E);
#pragma unroll
      for (int j = 0; j < PER; ++j) Ef[threadIdx.x + j * NT] = (float)(v[j] - c);
    }
    __syncthreads();
  } else {
    // a derivative channel (FP32, the engine's buffer): the plane arrives in
    // shared memory by one bulk copy
    __shared__ __align__(8) uint64_t bar;
    if (!bulk_load(E, src, sizeof(float) * NY * NZ, &bar, err)) return;
  }
  {
    // z, first half from the real plane in shared memory: task (y, n2)
    // takes the pairs E[y * M + BZ n1 + n2]
    constexpr int H0 = cdiv(P::T_Z_NAT, NT);
    cpx h0[H0][AZ];
#pragma unroll
    for (int j = 0; j < H0; ++j) {
      const int t = threadIdx.x + j * NT;
      if (t < P::T_Z_NAT) {
        const int n2 = t % BZ, y = t / BZ;
#pragma unroll
        for (int n1 = 0; n1 < AZ; ++n1) h0[j][n1] = E[y * M + BZ * n1 + n2];
        fft::nat_in<M, false>(h0[j], n2, tz);
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < H0; ++j) {
      const int t = threadIdx.x + j * NT;
      if (t < P::T_Z_NAT) {
        const int n2 = t % BZ, y = t / BZ;
#pragma unroll
        for (int k1 = 0; k1 < AZ; ++k1) E[y * EZ + n2 * EZS + k1] = h0[j][k1];
      }
    }
  }
  __syncthreads();
  // z, second half: task (y, k1) -> Z_y[kz = k1 + AZ k2]
  constexpr int H1 = cdiv(P::T_Z_SPEC, NT);
  cpx h1[H1][BZ];
#pragma unroll
  for (int j = 0; j < H1; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Z_SPEC) {
      const int k1 = t % AZ, y = t / AZ;
#pragma unroll
      for (int n2 = 0; n2 < BZ; ++n2) h1[j][n2] = E[y * EZ + n2 * EZS + k1];
      fft::nat_out<M, false>(h1[j]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < H1; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Z_SPEC) {
      const int k1 = t % AZ, y = t / AZ;
#pragma unroll
      for (int k2 = 0; k2 < BZ; ++k2) E[y * ER + k1 + AZ * k2] = h1[j][k2];
    }
  }
  __syncthreads();
  // y, first half: task (kz, n2) takes rows y = BY n1 + n2 of column kz
  constexpr int H2 = cdiv(P::T_Y_NAT, NT);
  cpx h2[H2][AY];
#pragma unroll
  for (int j = 0; j < H2; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Y_NAT) {
      const int kz = t % M, n2 = t / M;
#pragma unroll
      for (int n1 = 0; n1 < AY; ++n1) h2[j][n1] = E[(BY * n1 + n2) * ER + kz];
      fft::nat_in<NY, false>(h2[j], n2, ty);
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < H2; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Y_NAT) {
      const int kz = t % M, n2 = t / M;
#pragma unroll
      for (int k1 = 0; k1 < AY; ++k1) E[(n2 * AY + k1) * EY + kz] = h2[j][k1];
    }
  }
  __syncthreads();
  cpx* dst = out + ((long long)b * nseq + sq) * p.Nk + (long long)ix * NY * LD;
  // y, second half per mirror unit (fft::mirror_unit): the thread takes a
  // task and the task holding its elements' mirrors and post-processes
  // both from registers, with no further exchange
  for (int u = threadIdx.x; u < P::T_Y_SPEC / 2; u += NT) {
    const fft::MirrorUnit mu = fft::mirror_unit(u, M, AY);
    cpx za[BY], zb[BY];
#pragma unroll
    for (int n2 = 0; n2 < BY; ++n2) {
      za[n2] = E[(n2 * AY + mu.k1A) * EY + mu.kzA];
      zb[n2] = E[(n2 * AY + mu.k1B) * EY + mu.kzB];
    }
    fft::nat_out<NY, false>(za);
    fft::nat_out<NY, false>(zb);
    auto post = [&](const cpx(&zt)[BY], const cpx(&zo)[BY], int k1, int kz) {
#pragma unroll
      for (int k2 = 0; k2 < BY; ++k2) {
        const int ky = k1 + AY * k2;
        // the mirror: element mirror_k2(k1, k2) of the partner task
        const cpx m0 = mu.self ? zt[(BY - k2) % BY] : zo[(BY - k2) % BY];
        const cpx m1 = mu.self ? zt[BY - 1 - k2] : zo[BY - 1 - k2];
        const cpx zm = k1 == 0 ? m0 : m1;
        if (kz == 0) {
          cpx x0, xM;
          fft::r2c_post_2d_dc(zt[k2], zm, x0, xM);
          dst[ky * LD] = x0;
          dst[ky * LD + M] = xM;
        } else {
          dst[ky * LD + kz] = fft::r2c_post_2d(zt[k2], zm, t2[kz]);
        }
      }
    };
    post(za, zb, mu.k1A, mu.kzA);
    post(zb, za, mu.k1B, mu.kzB);
  }
}

// Inverse plane pass of one half spectrum (NY x (NZ/2 + 1), natural order):
// the C2R of its Hermitian projection, unnormalised.  EPI = false: written
// as a real FP32 channel.  EPI = true: the back-convolved force of species
// blockIdx.y, added to the FP64 force with the epilogue constant
// (force_s += hs dV - mu_s dV + the DC split term); the CTA of plane 0,
// species 0 of each problem also reduces the pointwise partials into the
// scalars (the pointwise kernel completed before this launch).
template <int NY, int NZ, bool EPI, bool MULTI, bool TENSOR, int NT = RPlane<NY, NZ>::NT>
__global__ void __launch_bounds__(NT)
    k_rplane_inv(EvalParams p, const cpx* __restrict__ in, int nseq, float* __restrict__ out_f,
                 double* __restrict__ force, const double* __restrict__ dbar, const __grid_constant__ MuArgs mu,
                 FinalArgs fin, int* err, int ix0, FftTables T) {
  pdl_trigger();
  pdl_wait();
  using P = RPlane<NY, NZ>;
  using L = Lay<MULTI, TENSOR>;
  constexpr int M = P::M, LD = P::LD, AY = P::AY, BY = P::BY, AZ = P::AZ, BZ = P::BZ;
  constexpr int EY = P::EY, ER = P::ER, EZS = P::EZS, EZ = P::EZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx* E = reinterpret_cast<cpx*>(smem_raw);
  cpx* ty = E + P::BUF;
  cpx* tz = ty + NY;
  cpx* t2 = tz + M;
  const int ix = ix0 + blockIdx.x, sq = blockIdx.y, b = blockIdx.z;  // planes ix0 ..
  __shared__ double s_const;
  if constexpr (EPI) {
    if (ix == 0 && sq == 0 && fin.scalars)
      reduce_final(fin.partials + (long long)b * fin.nblocks * p.n_terms, fin.nblocks, p, mu.mu[b], fin.err,
                   fin.scalars + b * kScalarCount);
    // the force plane is read at the end: start pulling it into L2 now
    const char* fp = reinterpret_cast<const char*>(force + ((long long)b * p.S + sq) * p.N + (long long)ix * NY * NZ);
    for (int off = threadIdx.x * 128; off < NY * NZ * 8; off += NT * 128)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(fp + off));
    if (threadIdx.x == 0) {
      double v = 0.0;
      const double* db = dbar + b * kMaxChannels;
#pragma unroll
      for (int c = 0; c < L::NFMT; ++c) v += chan_dc<MULTI, TENSOR>(c, sq, p) * db[c];
      s_const = v * p.dv - mu.mu[b][sq] * p.dv;
    }
  }
  plane_tables<NY, NZ, NT>(ty, tz, t2, T);
  __syncthreads();
  const cpx* src = in + ((long long)b * nseq + sq) * p.Nk + (long long)ix * NY * LD;
  // the half spectrum arrives in shared memory by one bulk copy: X[ky][kz]
  // at E[ky * LD + kz]
  __shared__ __align__(8) uint64_t bar;
  if (!bulk_load(E, src, sizeof(cpx) * NY * LD, &bar, err)) return;
  // y, first half: task (kz, k1) pre-processes X[ky = k1 + AY k2][kz] with
  // its mirror and starts the inverse y transform
  constexpr int H0 = cdiv(P::T_Y_SPEC, NT);
  cpx h0[H0][BY];
#pragma unroll
  for (int j = 0; j < H0; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Y_SPEC) {
      const int kz = t % M, k1 = t / M;
#pragma unroll
      for (int k2 = 0; k2 < BY; ++k2) {
        const int ky = k1 + AY * k2, km = (NY - ky) % NY;
        if (kz == 0)
          h0[j][k2] = fft::c2r_pre_2d_dc(E[ky * LD], E[km * LD], E[ky * LD + M], E[km * LD + M]);
        else
          h0[j][k2] = fft::c2r_pre_2d(E[ky * LD + kz], E[km * LD + (M - kz)], t2[kz]);
      }
      fft::spec_in<NY, true>(h0[j], k1, ty);
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < H0; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Y_SPEC) {
      const int kz = t % M, k1 = t / M;
#pragma unroll
      for (int n2 = 0; n2 < BY; ++n2) E[(n2 * AY + k1) * EY + kz] = h0[j][n2];
    }
  }
  __syncthreads();
  // y, second half: task (kz, n2) -> rows y = BY n1 + n2
  constexpr int H1 = cdiv(P::T_Y_NAT, NT);
  cpx h1[H1][AY];
#pragma unroll
  for (int j = 0; j < H1; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Y_NAT) {
      const int kz = t % M, n2 = t / M;
#pragma unroll
      for (int k1 = 0; k1 < AY; ++k1) h1[j][k1] = E[(n2 * AY + k1) * EY + kz];
      fft::spec_out<NY, true>(h1[j]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < H1; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Y_NAT) {
      const int kz = t % M, n2 = t / M;
#pragma unroll
      for (int n1 = 0; n1 < AY; ++n1) E[(BY * n1 + n2) * ER + kz] = h1[j][n1];
    }
  }
  __syncthreads();
  // z, first half: task (y, k1) takes Z_y[kz = k1 + AZ k2]
  constexpr int H2 = cdiv(P::T_Z_SPEC, NT);
  cpx h2[H2][BZ];
#pragma unroll
  for (int j = 0; j < H2; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Z_SPEC) {
      const int k1 = t % AZ, y = t / AZ;
#pragma unroll
      for (int k2 = 0; k2 < BZ; ++k2) h2[j][k2] = E[y * ER + k1 + AZ * k2];
      fft::spec_in<M, true>(h2[j], k1, tz);
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < H2; ++j) {
    const int t = threadIdx.x + j * NT;
    if (t < P::T_Z_SPEC) {
      const int k1 = t % AZ, y = t / AZ;
#pragma unroll
      for (int n2 = 0; n2 < BZ; ++n2) E[y * EZ + n2 * EZS + k1] = h2[j][n2];
    }
  }
  __syncthreads();
  // z, second half: task (y, n2) -> pairs n = BZ n1 + n2 of row y
  const long long plane_off = ((long long)b * (EPI ? p.S : nseq) + sq) * p.N + (long long)ix * NY * NZ;
  double cst = 0.0;
  if constexpr (EPI) cst = s_const;
  // a 16-byte aligned force takes each sample pair in one load and one store
  // (plane_off and 2 n are even)
  const bool pairs = EPI && (reinterpret_cast<uintptr_t>(force) & 15) == 0;
  for (int t = threadIdx.x; t < P::T_Z_NAT; t += NT) {
    const int n2 = t % BZ, y = t / BZ;
    cpx a[AZ];
#pragma unroll
    for (int k1 = 0; k1 < AZ; ++k1) a[k1] = E[y * EZ + n2 * EZS + k1];
    fft::spec_out<M, true>(a);
#pragma unroll
    for (int n1 = 0; n1 < AZ; ++n1) {
      const int n = BZ * n1 + n2;
      if constexpr (EPI) {
        double* f = force + plane_off + (long long)y * NZ + 2 * n;
        if (pairs) {
          double2 fv = *reinterpret_cast<const double2*>(f);
          fv.x = fv.x + (double)(2.0f * a[n1].x) * p.dv + cst;
          fv.y = fv.y + (double)(2.0f * a[n1].y) * p.dv + cst;
          *reinterpret_cast<double2*>(f) = fv;
        } else {  // the caller's buffer, 8-byte aligned only
          f[0] = f[0] + (double)(2.0f * a[n1].x) * p.dv + cst;
          f[1] = f[1] + (double)(2.0f * a[n1].y) * p.dv + cst;
        }
      } else {
        *reinterpret_cast<float2*>(out_f + plane_off + (long long)y * NZ + 2 * n) =
            make_float2(2.0f * a[n1].x, 2.0f * a[n1].y);
      }
    }
  }
}

// ----------------------------------------------------------- column pass

// Fused-path weight table, built once per engine: per species the |k|
// factors pre-scaled by 1/N, FP64-computed and rounded to FP32 -- w3, w2,
// fv, A/k^2, B -- then the mean-field weights (real) in FP32.  Layout
// [S][5][Nk] floats, then [M][Nk].
__host__ __device__ inline long long rweight_table_floats(const EvalParams& p) { return (5LL * p.S + p.M) * p.Nk; }

static __global__ void __launch_bounds__(256)
    k_build_rweights(EvalParams p, const double* __restrict__ mf_w, float* __restrict__ tab) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < p.Nk;
       idx += (long long)gridDim.x * blockDim.x) {
    const KIndex q = decode_k(p, idx);
    double kk[3], km[3], k, inv_k2;
    k_setup(p, q, kk, km, k, inv_k2);
    for (int s = 0; s < p.S; ++s) {
      const KW w = weight_kernels(k, p.R[s]);
      float* t = tab + 5LL * s * p.Nk + idx;
      t[0] = (float)(w.w3 * p.inv_n);
      t[p.Nk] = (float)(w.w2 * p.inv_n);
      t[2 * p.Nk] = (float)(w.fv * p.inv_n);
      t[3 * p.Nk] = (float)(w.A * inv_k2 * p.inv_n);
      t[4 * p.Nk] = (float)(w.B * p.inv_n);
    }
    for (int m = 0; m < p.M; ++m) tab[(5LL * p.S + m) * p.Nk + idx] = (float)mf_w[m * p.Nk + idx];
  }
}

// The symmetrised k-space factors of one element.  On the self-conjugate
// planes (kz = 0 and kz = nz/2: `proj` columns) the channel weights become
// W'(k) = (W(k) + conj W(k_m)) / 2 with the mirror k_m = (-kx, -ky, kz),
// except that a Nyquist x or y index is its own mirror.  With s_a = -1 for
// a mirrored component and +1 for an unmirrored one (z always, Nyquist x or
// y), an odd channel k_a keeps its weight iff s_a = -1 and a tensor cross
// term k_a k_b iff s_a = s_b; every other weight is unchanged.
struct RKv {
  float k[3];   // the wavevector
  float o[3];   // odd-channel masks
  float cxy, cxz, cyz;  // tensor cross-term masks
};

__device__ __forceinline__ RKv rk_element(float kx, bool xnyq, float ky, bool ynyq, float kz, bool proj) {
  RKv v;
  v.k[0] = kx;
  v.k[1] = ky;
  v.k[2] = kz;
  v.o[0] = (!proj || !xnyq) ? 1.0f : 0.0f;
  v.o[1] = (!proj || !ynyq) ? 1.0f : 0.0f;
  v.o[2] = proj ? 0.0f : 1.0f;
  v.cxy = (!proj || xnyq == ynyq) ? 1.0f : 0.0f;
  v.cxz = (!proj || xnyq) ? 1.0f : 0.0f;
  v.cyz = (!proj || ynyq) ? 1.0f : 0.0f;
  return v;
}

__device__ __forceinline__ float rk_cross(const RKv& v, int i, int j) {
  if (i == j) return 1.0f;
  if (i + j == 1) return v.cxy;
  if (i + j == 2) return v.cxz;
  return v.cyz;
}

// Weight of FMT channel c for species s (c uniform across the block): the
// channel is w rho_s, or i w rho_s when `odd`.  weights.hpp:163-179 with the
// Rosenfeld scalings of hard_sphere.hpp:80-85, as chan_weight.
template <bool MULTI, bool TENSOR>
__device__ __forceinline__ float rk_weight(int c, const float* __restrict__ ts, long long Nk, const RKv& v,
                                           float i4r, float i4r2, bool& odd) {
  using L = Lay<MULTI, TENSOR>;
  odd = false;
  if (c == L::ETA) return ts[0];
  if (c == L::N2) return ts[Nk];
  if (MULTI && c == L::N1) return ts[Nk] * i4r;
  if (MULTI && c == L::N0) return ts[Nk] * i4r2;
  if (c >= L::V1 && c < L::V1 + 3) {
    odd = true;
    const int a = c - L::V1;
    return ts[2 * Nk] * (v.k[a] * v.o[a]);
  }
  if (MULTI && c >= L::V0 && c < L::V0 + 3) {
    odd = true;
    const int a = c - L::V0;
    return (ts[2 * Nk] * (v.k[a] * v.o[a])) * i4r;
  }
  const int t = c - L::T;
  const int i = tchan_i(t), j = tchan_j(t);
  const float kij = v.k[i] * v.k[j] * rk_cross(v, i, j);
  return (i == j) ? ts[3 * Nk] * kij + ts[4 * Nk] : ts[3 * Nk] * kij;
}

template <int NX>
struct RCol {
  using SX = fft::Split<NX>;
  static constexpr int AX = SX::A, BX = SX::B;
  static constexpr int NT = 256;
};

// Shared memory of a column kernel with TQ columns: the x twiddles, two
// exchange buffers and `nkeep` natural-order spectra (rho_k of every species
// forward, the force accumulators backward), each NX x TQ.
__host__ __device__ inline size_t rcol_smem(int nx, int tq, int nkeep) {
  return sizeof(cpx) * ((size_t)nx + (size_t)(2 + nkeep) * nx * tq);
}

// Per-column constants of in-plane index q.
struct RColumn {
  float ky, kz;
  bool ynyq, proj, valid;
};

__device__ __forceinline__ RColumn rk_column(const EvalParams& p, long long q, float dky, float dkz) {
  RColumn c;
  const long long plane = (long long)p.ny * p.nzh;
  c.valid = q < plane;
  const int iy = c.valid ? (int)(q / p.nzh) : 0;
  const int iz = c.valid ? (int)(q - (long long)iy * p.nzh) : 0;
  c.ky = dky * (float)(iy <= p.ny / 2 ? iy : iy - p.ny);
  c.kz = dkz * (float)iz;
  c.ynyq = (p.ny % 2 == 0) && iy == p.ny / 2;
  c.proj = (iz == 0) || (((p.nz & 1) == 0) && iz == p.nz / 2);
  return c;
}

// Forward transform along x of one array's column tile: the natural-order
// spectrum of tile column q, row kx, goes to spec[kx * TQ + q].  dc (or
// null): real parts added to in-plane column 0 before the transform (the
// plane-mean correction of the split rho, see rk_dc_column).
template <int NX, int TQ>
__device__ __forceinline__ void col_forward(const cpx* __restrict__ src, long long plane, long long q0, cpx* E,
                                            cpx* spec, const cpx* tx, const float* dc = nullptr) {
  using C = RCol<NX>;
  constexpr int AX = C::AX, BX = C::BX, NT = C::NT;
#pragma unroll 1
  for (int t = threadIdx.x; t < TQ * BX; t += NT) {
    const int q = t % TQ, n2 = t / TQ;
    const bool ok = q0 + q < plane;
    cpx a[AX];
#pragma unroll
    for (int n1 = 0; n1 < AX; ++n1) a[n1] = ok ? src[(BX * n1 + n2) * plane + q0 + q] : cpx{0.0f, 0.0f};
    if (dc && q0 + q == 0) {
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1].x += dc[BX * n1 + n2];
    }
    fft::nat_in<NX, false>(a, n2, tx);
#pragma unroll
    for (int k1 = 0; k1 < AX; ++k1) E[(n2 * AX + k1) * TQ + q] = a[k1];
  }
  __syncthreads();
#pragma unroll 1
  for (int t = threadIdx.x; t < TQ * AX; t += NT) {
    const int q = t % TQ, k1 = t / TQ;
    cpx bv[BX];
#pragma unroll
    for (int n2 = 0; n2 < BX; ++n2) bv[n2] = E[(n2 * AX + k1) * TQ + q];
    fft::nat_out<NX, false>(bv);
#pragma unroll
    for (int k2 = 0; k2 < BX; ++k2) spec[(k1 + AX * k2) * TQ + q] = bv[k2];
  }
}

// Inverse transform along x of the natural-order spectrum whose values
// kx = k1 + AX k2 (k2 < BX) of column q values(k1, q, bv) fills (called by
// the thread that owns them in col_forward's second half), stored to dst
// column q0 + q.
template <int NX, int TQ, class V>
__device__ __forceinline__ void col_inverse(V&& values, cpx* E, const cpx* tx, cpx* __restrict__ dst,
                                            long long plane, long long q0) {
  using C = RCol<NX>;
  constexpr int AX = C::AX, BX = C::BX, NT = C::NT;
#pragma unroll 1
  for (int t = threadIdx.x; t < TQ * AX; t += NT) {
    const int q = t % TQ, k1 = t / TQ;
    cpx bv[BX];
    values(k1, q, bv);
    fft::spec_in<NX, true>(bv, k1, tx);
#pragma unroll
    for (int n2 = 0; n2 < BX; ++n2) E[(n2 * AX + k1) * TQ + q] = bv[n2];
  }
  __syncthreads();
#pragma unroll 1
  for (int t = threadIdx.x; t < TQ * BX; t += NT) {
    const int q = t % TQ, n2 = t / TQ;
    cpx a[AX];
#pragma unroll
    for (int k1 = 0; k1 < AX; ++k1) a[k1] = E[(n2 * AX + k1) * TQ + q];
    fft::spec_out<NX, true>(a);
    if (q0 + q < plane) {
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) dst[(BX * n1 + n2) * plane + q0 + q] = a[n1];
    }
  }
}

// The species means and the plane-mean correction of the split rho.  The
// plane pass transformed rho - m_x (m_x: plane x's mean, in pmean); the
// channels are built on rho - m with m the species mean (the FP64 offset
// the pointwise kernel adds back), so in-plane column (ky, kz) = (0, 0)
// gets (m_x - m) NY NZ added before its x transform: small, the plane
// means' own fluctuation.  Run by the CTA that holds column 0 (uniformly);
// writes m to mean_out for the later stages.  dc: S x NX floats in shared
// memory.
template <int NX>
__device__ __forceinline__ void rk_dc_column(const EvalParams& p, const double* __restrict__ pmean, int b,
                                             double* __restrict__ mean_out, float* dc) {
  __shared__ double s_m[kMaxSpecies];
  const int S = p.S;
  if (threadIdx.x < S) {
    const double* pm = pmean + ((long long)b * S + threadIdx.x) * NX;
    double m = 0.0;
    for (int x = 0; x < NX; ++x) m += pm[x];
    m /= (double)NX;
    s_m[threadIdx.x] = m;
    mean_out[b * kMaxSpecies + threadIdx.x] = m;
  }
  __syncthreads();
  const double nyz = (double)p.ny * (double)p.nz;
  for (int i = threadIdx.x; i < S * NX; i += blockDim.x) {
    const int s = i / NX, x = i % NX;
    dc[s * NX + x] = (float)((pmean[((long long)b * S + s) * NX + x] - s_m[s]) * nyz);
  }
  __syncthreads();
}

// Column pass of the forward stage: rho_k along x for every species, then
// for every channel its k-space product and the inverse x transform.  Tile:
// in-plane indices q0 .. q0 + TQ - 1 of all NX planes.  The two exchange
// buffers alternate, so one barrier per transform suffices.
template <int NX, int TQ, bool MULTI, bool TENSOR>
__global__ void __launch_bounds__(256, 2)
    k_rcol_fwd(EvalParams p, const cpx* __restrict__ prho, const double* __restrict__ pmean,
               double* __restrict__ mean_out, const float* __restrict__ wtab, cpx* __restrict__ q_out, FftTables T) {
  pdl_trigger();
  pdl_wait();
  using L = Lay<MULTI, TENSOR>;
  constexpr int NT = RCol<NX>::NT, TILE = NX * TQ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx* tx = reinterpret_cast<cpx*>(smem_raw);
  cpx* Eb = tx + NX;
  cpx* R = Eb + 2 * TILE;
  const int S = p.S, C = p.n_chan;
  const long long plane = (long long)p.ny * p.nzh, Nk = p.Nk;
  const int b = blockIdx.y;
  const long long q0 = (long long)blockIdx.x * TQ;
  __shared__ float s_dc[kMaxSpecies * NX];
  for (int i = threadIdx.x; i < NX; i += NT) tx[i] = T.tx[i];
  if (blockIdx.x == 0) rk_dc_column<NX>(p, pmean, b, mean_out, s_dc);
  __syncthreads();
  int buf = 0;
  for (int s = 0; s < S; ++s) {
    col_forward<NX, TQ>(prho + ((long long)b * S + s) * Nk, plane, q0, Eb + buf * TILE, R + (size_t)s * TILE, tx,
                        blockIdx.x == 0 ? s_dc + s * NX : nullptr);
    buf ^= 1;
  }
  const float dkx = (float)p.dkx, dky = (float)p.dky, dkz = (float)p.dkz;
  float i4r[kMaxSpecies], i4r2[kMaxSpecies];
#pragma unroll
  for (int s = 0; s < kMaxSpecies; ++s) {
    i4r[s] = (float)p.inv4piR[s];
    i4r2[s] = (float)p.inv4piR2[s];
  }
  for (int c = 0; c < C; ++c) {
    // mean-field channel c: w * rho of species mf_sp (weight table mf_m)
    int mf_m = -1, mf_sp = 0;
    for (int m = 0; m < p.M; ++m) {
      if (c == p.mf_chan_j[m]) mf_m = m, mf_sp = p.mf_j[m];
      if (c == p.mf_chan_i[m]) mf_m = m, mf_sp = p.mf_i[m];
    }
    auto values = [&](int k1, int q, cpx* bv) {
      const RColumn col = rk_column(p, q0 + q, dky, dkz);
#pragma unroll
      for (int k2 = 0; k2 < RCol<NX>::BX; ++k2) {
        const int kx = k1 + RCol<NX>::AX * k2;
        const long long kidx = (long long)kx * plane + q0 + q;
        cpx acc{0.0f, 0.0f};
        if (col.valid) {
          if (mf_m >= 0) {
            const float w = wtab[(5LL * S + mf_m) * Nk + kidx];
            const cpx r = R[(size_t)mf_sp * TILE + kx * TQ + q];
            acc = cpx{w * r.x, w * r.y};
          } else {
            // (NX equals p.nx here; the constant lets the compiler fold the
            // element's sign and Nyquist tests)
            const bool xnyq = (NX % 2 == 0) && kx == NX / 2;
            const RKv v = rk_element(dkx * (float)(kx <= NX / 2 ? kx : kx - NX), xnyq, col.ky, col.ynyq, col.kz,
                                     col.proj);
#pragma unroll
            for (int s = 0; s < (MULTI ? kMaxSpecies : 1); ++s) {
              if (s < S) {
                bool odd;
                const float w = rk_weight<MULTI, TENSOR>(c, wtab + 5LL * s * Nk + kidx, Nk, v, i4r[s], i4r2[s], odd);
                const cpx r = R[(size_t)s * TILE + kx * TQ + q];
                if (odd) {
                  acc.x -= w * r.y;
                  acc.y += w * r.x;
                } else {
                  acc.x += w * r.x;
                  acc.y += w * r.y;
                }
              }
            }
          }
        }
        bv[k2] = acc;
      }
    };
    col_inverse<NX, TQ>(values, Eb + buf * TILE, tx, q_out + ((long long)b * C + c) * Nk, plane, q0);
    buf ^= 1;
  }
}

// Column pass of the backward stage: every derivative channel along x, the
// back-convolution F_s = sum_c conj(W'_cs) D_c accumulated per element by
// the thread that owns it, then the inverse x transform of each F_s.
template <int NX, int TQ, bool MULTI, bool TENSOR>
__global__ void __launch_bounds__(256, 2)
    k_rcol_bwd(EvalParams p, const cpx* __restrict__ pd, const float* __restrict__ wtab, cpx* __restrict__ pf,
               FftTables T) {
  pdl_trigger();
  pdl_wait();
  using L = Lay<MULTI, TENSOR>;
  constexpr int NF = L::NFMT, NT = RCol<NX>::NT, TILE = NX * TQ;
  constexpr int AX = RCol<NX>::AX, BX = RCol<NX>::BX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx* tx = reinterpret_cast<cpx*>(smem_raw);
  cpx* Eb = tx + NX;
  cpx* F = Eb + 2 * TILE;  // S natural-order force spectra
  const int S = p.S;
  const long long plane = (long long)p.ny * p.nzh, Nk = p.Nk;
  const int b = blockIdx.y;
  const long long q0 = (long long)blockIdx.x * TQ;
  for (int i = threadIdx.x; i < NX; i += NT) tx[i] = T.tx[i];
  const float dkx = (float)p.dkx, dky = (float)p.dky, dkz = (float)p.dkz;
  float i4r[kMaxSpecies], i4r2[kMaxSpecies];
#pragma unroll
  for (int s = 0; s < kMaxSpecies; ++s) {
    i4r[s] = (float)p.inv4piR[s];
    i4r2[s] = (float)p.inv4piR2[s];
  }
  __syncthreads();
  int buf = 0;
  for (int c = 0; c < NF; ++c) {
    cpx* E = Eb + buf * TILE;
    const cpx* src = pd + ((long long)b * NF + c) * Nk;
#pragma unroll 1
    for (int t = threadIdx.x; t < TQ * BX; t += NT) {
      const int q = t % TQ, n2 = t / TQ;
      const bool ok = q0 + q < plane;
      cpx a[AX];
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = ok ? src[(BX * n1 + n2) * plane + q0 + q] : cpx{0.0f, 0.0f};
      fft::nat_in<NX, false>(a, n2, tx);
#pragma unroll
      for (int k1 = 0; k1 < AX; ++k1) E[(n2 * AX + k1) * TQ + q] = a[k1];
    }
    __syncthreads();
#pragma unroll 1
    for (int t = threadIdx.x; t < TQ * AX; t += NT) {
      const int q = t % TQ, k1 = t / TQ;
      cpx d[BX];
#pragma unroll
      for (int n2 = 0; n2 < BX; ++n2) d[n2] = E[(n2 * AX + k1) * TQ + q];
      fft::nat_out<NX, false>(d);
      const RColumn col = rk_column(p, q0 + q, dky, dkz);
#pragma unroll
      for (int k2 = 0; k2 < BX; ++k2) {
        const int kx = k1 + AX * k2;
        const long long kidx = (long long)kx * plane + q0 + q;
        const bool xnyq = (NX % 2 == 0) && kx == NX / 2;
        const RKv v = rk_element(dkx * (float)(kx <= NX / 2 ? kx : kx - NX), xnyq, col.ky, col.ynyq, col.kz, col.proj);
#pragma unroll
        for (int s = 0; s < (MULTI ? kMaxSpecies : 1); ++s) {
          if (s < S) {
            cpx add{0.0f, 0.0f};
            if (col.valid) {
              bool odd;
              const float w = rk_weight<MULTI, TENSOR>(c, wtab + 5LL * s * Nk + kidx, Nk, v, i4r[s], i4r2[s], odd);
              // conj(i w) D = -i w D for an odd channel
              add = odd ? cpx{w * d[k2].y, -w * d[k2].x} : cpx{w * d[k2].x, w * d[k2].y};
            }
            cpx& f = F[(size_t)s * TILE + kx * TQ + q];
            f = (c == 0) ? add : f + add;
          }
        }
      }
    }
    buf ^= 1;
  }
  for (int s = 0; s < S; ++s) {
    auto values = [&](int k1, int q, cpx* bv) {
#pragma unroll
      for (int k2 = 0; k2 < BX; ++k2) bv[k2] = F[(size_t)s * TILE + (k1 + AX * k2) * TQ + q];
    };
    col_inverse<NX, TQ>(values, Eb + buf * TILE, tx, pf + ((long long)b * S + s) * Nk, plane, q0);
    buf ^= 1;
  }
}

// ------------------------------------------- single-species column passes

// One species: the thread of spectrum task (q, k1) keeps its BX elements'
// |k| factors and rho_k (forward) or force accumulators (backward) in
// registers for the whole pass.  One spectrum task per thread (NT = TQ *
// AX); the first TQ * BX threads also run the natural-order half of each
// transform.  Natural-order task (q, n2) and spectrum task (q, k1) of a
// thread share its column q = t % TQ.
template <int NX, int TQ>
struct RCol1 {
  using SX = fft::Split<NX>;
  static constexpr int AX = SX::A, BX = SX::B;
  static constexpr int NT = TQ * AX;
  static constexpr int TILE = NX * TQ;
  static constexpr int KN = NX / 2;                   // the x Nyquist element
  static constexpr int K1N = KN % AX, K2N = KN / AX;  // its spectrum task and slot
  // AX = 2 BX (128, 32): the second half of an inverse transform runs on
  // every thread, two per natural-order task with half of its samples each
  static constexpr bool SPLIT_OUT = AX == 2 * BX;
  static_assert(NX % 2 == 0, "even column lengths only");
};

// Forward: tx, two exchange buffers and two kept transforms of NX x TQ;
// backward: tx, two exchange buffers and four load buffers.
__host__ __device__ inline size_t rcol1_smem(int nx, int tq) { return sizeof(cpx) * ((size_t)nx + 4ull * nx * tq); }
__host__ __device__ inline size_t rcol1_smem_bwd(int nx, int tq) {
  return sizeof(cpx) * ((size_t)nx + 6ull * nx * tq);
}

// The |k| factors of a task's elements (zero for columns past the plane).
template <int BX>
struct RTab {
  float w3[BX], w2[BX], fv[BX], a[BX];
};

template <int NX, int TQ>
__device__ __forceinline__ RTab<RCol1<NX, TQ>::BX> rk_task_table(const float* __restrict__ wtab, long long Nk,
                                                                   long long plane, long long col0, int k1,
                                                                   bool valid) {
  constexpr int AX = RCol1<NX, TQ>::AX, BX = RCol1<NX, TQ>::BX;
  RTab<BX> t;
#pragma unroll
  for (int k2 = 0; k2 < BX; ++k2) {
    const long long kidx = (long long)(k1 + AX * k2) * plane + col0;
    t.w3[k2] = valid ? wtab[kidx] : 0.0f;
    t.w2[k2] = valid ? wtab[Nk + kidx] : 0.0f;
    t.fv[k2] = valid ? wtab[2 * Nk + kidx] : 0.0f;
    t.a[k2] = valid ? wtab[3 * Nk + kidx] : 0.0f;
  }
  return t;
}

// Element kx of a column (NX = p.nx: the compile-time length folds the sign
// and Nyquist tests of the unrolled elements).
template <int NX>
__device__ __forceinline__ RKv rk_task_element(const EvalParams&, int kx, float dkx, const RColumn& col) {
  const bool xnyq = (NX % 2 == 0) && kx == NX / 2;
  return rk_element(dkx * (float)(kx <= NX / 2 ? kx : kx - NX), xnyq, col.ky, col.ynyq, col.kz, col.proj);
}

// Column bases.  Along one column (ky, kz fixed) every FMT weight of one
// species (weights.hpp:163-179; channel = W rho) is a few kx-dependent
// factors times column constants:
//   W_vy = i fv ky o_y,  W_vz = i fv kz o_z,
//   W_Txy = a kx ky c_xy,  W_Txz = a kx kz c_xz,  W_Tyz = a ky kz c_yz,
// and, with the trace identity a k^2 + 3 b = w2 of the tensor weight
// a k_i k_j + b delta_ij,
//   W_Txx = (2/3) a kx^2 + w2 / 3 - (ky^2 + kz^2) / 3 a,
//   W_Tyy = -(1/3) a kx^2 + w2 / 3 + (2 ky^2 - kz^2) / 3 a.
// So one x transform per basis serves every channel of a column:
//   w3, w2, i fv kx o_x, i fv, a kx c_xy, a, a kx^2
// (the first four without the tensor): 7 transforms for 10 channels.  The
// Hermitian-projection masks o_x and c_xy depend on kx only at the x
// Nyquist element.  c_xz equals c_xy on every column with kz != 0 except
// those of the kz = nz/2 plane with ky off Nyquist ("special" columns),
// where c_xz keeps only the x Nyquist element, whose transform is the
// single term c (-1)^x.
enum : int { kBW3 = 0, kBW2 = 1, kBVX = 2, kBV = 3, kBTX = 4, kBTA = 5, kBTXX = 6 };

// The real factors of basis j at the BX elements of a task; returns `odd`
// (the basis is i w).
template <int NX, int TQ>
__device__ __forceinline__ bool rk_basis_weights(int j, const RTab<RCol1<NX, TQ>::BX>& t, const EvalParams& p,
                                                 int k1, float dkx, const RColumn& col,
                                                 float (&w)[RCol1<NX, TQ>::BX]) {
  constexpr int AX = RCol1<NX, TQ>::AX, BX = RCol1<NX, TQ>::BX;
  // (j is uniform: one branch per basis; only the kx bases form kx)
  if (j == kBW3 || j == kBW2 || j == kBV || j == kBTA) {
#pragma unroll
    for (int k2 = 0; k2 < BX; ++k2)
      w[k2] = j == kBW3 ? t.w3[k2] : j == kBW2 ? t.w2[k2] : j == kBV ? t.fv[k2] : t.a[k2];
  } else {
#pragma unroll
    for (int k2 = 0; k2 < BX; ++k2) {
      const RKv v = rk_task_element<NX>(p, k1 + AX * k2, dkx, col);
      const float kx = v.k[0];
      if (j == kBVX)
        w[k2] = t.fv[k2] * (kx * v.o[0]);
      else if (j == kBTX)
        w[k2] = t.a[k2] * (kx * v.cxy);
      else
        w[k2] = t.a[k2] * (kx * kx);
    }
  }
  return j == kBVX || j == kBV;
}

// Column constants of the basis combinations (zero past the plane).
struct RColK {
  float ky, kz;
  float vy, vz, yz;  // ky o_y, kz o_z, ky kz c_yz
  bool special;      // kz = nz/2 plane, ky off Nyquist
};

__device__ __forceinline__ RColK rk_colk(const RColumn& c) {
  RColK r;
  r.ky = c.valid ? c.ky : 0.0f;
  r.kz = c.valid ? c.kz : 0.0f;
  r.vy = (!c.proj || !c.ynyq) ? r.ky : 0.0f;
  r.vz = c.proj ? 0.0f : r.kz;
  r.yz = (!c.proj || c.ynyq) ? r.ky * r.kz : 0.0f;
  r.special = c.valid && c.proj && c.kz != 0.0f && !c.ynyq;
  return r;
}

// Inverse x transform of the task values bv (this thread's spectrum task)
// through exchange buffer E.  The second half hands the samples of
// natural-order task (q, n2) to emit(v, n1_0, dn1, n2): v[i] is sample
// x = BX (n1_0 + i dn1) + n2 of column q.  With SPLIT_OUT the two threads
// t and t + TQ BX of a task compute its even and odd n1 (dft_half), else
// the first TQ BX threads compute all AX.  The caller alternates E between
// two buffers.
template <int NX, int TQ, class Emit>
__device__ __forceinline__ void col1_inverse_emit(cpx (&bv)[RCol1<NX, TQ>::BX], int q, int k1, cpx* E,
                                                  const cpx* tx, Emit&& emit) {
  using C = RCol1<NX, TQ>;
  constexpr int AX = C::AX, BX = C::BX;
  fft::spec_in<NX, true>(bv, k1, tx);
#pragma unroll
  for (int n2 = 0; n2 < BX; ++n2) E[(n2 * AX + k1) * TQ + q] = bv[n2];
  __syncthreads();
  const int t = threadIdx.x;
  if constexpr (C::SPLIT_OUT) {
    const int h = t / (TQ * BX), n2 = (t / TQ) % BX;
    cpx a[AX];
#pragma unroll
    for (int kk = 0; kk < AX; ++kk) a[kk] = E[(n2 * AX + kk) * TQ + q];
    cpx v[AX / 2];
    fft::dft_half<AX, true>(a, h, v);
    emit(v, h, 2, n2);
  } else if (t < TQ * BX) {
    const int n2 = t / TQ;
    cpx a[AX];
#pragma unroll
    for (int kk = 0; kk < AX; ++kk) a[kk] = E[(n2 * AX + kk) * TQ + q];
    fft::spec_out<NX, true>(a);
    emit(a, 0, 1, n2);
  }
}

template <int NX, int TQ>
__device__ __forceinline__ void col1_inverse(cpx (&bv)[RCol1<NX, TQ>::BX], int q, int k1, cpx* E, const cpx* tx,
                                             cpx* __restrict__ dst, long long plane, long long q0) {
  constexpr int BX = RCol1<NX, TQ>::BX;
  col1_inverse_emit<NX, TQ>(bv, q, k1, E, tx, [&](const auto& v, int n1_0, int dn1, int n2) {
    constexpr int K = std::extent_v<std::remove_reference_t<decltype(v)>>;
    if (q0 + q < plane) {
#pragma unroll
      for (int i = 0; i < K; ++i) dst[(BX * (n1_0 + i * dn1) + n2) * plane + q0 + q] = v[i];
    }
  });
}

// Forward x transform of one array's column tile into this thread's task
// values (natural-order spectrum elements k1 + AX k2 of column q).
template <int NX, int TQ>
__device__ __forceinline__ void col1_forward(const cpx* __restrict__ src, long long plane, long long q0, int q, int k1,
                                             cpx* E, const cpx* tx, cpx (&out)[RCol1<NX, TQ>::BX],
                                             const float* dc = nullptr) {
  using C = RCol1<NX, TQ>;
  constexpr int AX = C::AX, BX = C::BX;
  const int t = threadIdx.x;
  if (t < TQ * BX) {
    const int n2 = t / TQ;
    const bool ok = q0 + q < plane;
    cpx a[AX];
#pragma unroll
    for (int n1 = 0; n1 < AX; ++n1) a[n1] = ok ? src[(BX * n1 + n2) * plane + q0 + q] : cpx{0.0f, 0.0f};
    if (dc && q0 + q == 0) {
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1].x += dc[BX * n1 + n2];
    }
    fft::nat_in<NX, false>(a, n2, tx);
#pragma unroll
    for (int kk = 0; kk < AX; ++kk) E[(n2 * AX + kk) * TQ + q] = a[kk];
  }
  __syncthreads();
#pragma unroll
  for (int n2 = 0; n2 < BX; ++n2) out[n2] = E[(n2 * AX + k1) * TQ + q];
  fft::nat_out<NX, false>(out);
}

// Forward column pass: rho along x, then one inverse x transform per basis
// (and per mean-field channel), each written out as the channels it
// serves.  The w2 and a transforms stay in shared memory (each thread
// reads back only its own samples) until the a kx^2 basis combines them
// into T_xx and T_yy.
template <int NX, int TQ, bool TENSOR>
__global__ void __launch_bounds__(RCol1<NX, TQ>::NT, 2)
    k_rcol_fwd1(EvalParams p, const cpx* __restrict__ prho, const double* __restrict__ pmean,
                double* __restrict__ mean_out, const float* __restrict__ wtab, cpx* __restrict__ q_out, FftTables T) {
  pdl_trigger();
  pdl_wait();
  using L = Lay<false, TENSOR>;
  using C = RCol1<NX, TQ>;
  constexpr int AX = C::AX, BX = C::BX, NT = C::NT, TILE = C::TILE;
  constexpr int NB = TENSOR ? 7 : 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx* tx = reinterpret_cast<cpx*>(smem_raw);
  cpx* Eb = tx + NX;
  cpx* S1 = Eb + 2 * TILE;  // the w2 transform
  cpx* S2 = S1 + TILE;      // the a transform
  __shared__ cpx s_nyq[TQ];  // a kx rho at the x Nyquist element of each column
  __shared__ float s_dc[NX];
  const long long plane = (long long)p.ny * p.nzh, Nk = p.Nk;
  const int b = blockIdx.y;
  const long long q0 = (long long)blockIdx.x * TQ;
  const int t = threadIdx.x;
  const int q = t % TQ, k1 = t / TQ;
  for (int i = t; i < NX; i += NT) tx[i] = T.tx[i];
  const RColumn col = rk_column(p, q0 + q, (float)p.dky, (float)p.dkz);
  const RColK ck = rk_colk(col);
  const RTab<BX> tab = rk_task_table<NX, TQ>(wtab, Nk, plane, q0 + q, k1, col.valid);
  const float dkx = (float)p.dkx;
  if (blockIdx.x == 0) rk_dc_column<NX>(p, pmean, b, mean_out, s_dc);
  __syncthreads();
  cpx r[BX];
  col1_forward<NX, TQ>(prho + (long long)b * Nk, plane, q0, q, k1, Eb, tx, r, blockIdx.x == 0 ? s_dc : nullptr);
  int buf = 1;
  cpx* out = q_out + (long long)b * p.n_chan * Nk + q0 + q;
  const float third = 1.0f / 3.0f;
#pragma unroll 1
  for (int j = 0; j < NB; ++j) {
    float w[BX];
    const bool odd = rk_basis_weights<NX, TQ>(j, tab, p, k1, dkx, col, w);
    cpx bv[BX];
#pragma unroll
    for (int k2 = 0; k2 < BX; ++k2) bv[k2] = odd ? cpx{-w[k2] * r[k2].y, w[k2] * r[k2].x} : scale(r[k2], w[k2]);
    if (TENSOR && j == kBTX && k1 == C::K1N) s_nyq[q] = scale(r[C::K2N], tab.a[C::K2N] * (dkx * (float)C::KN));
    // the channels of basis j: c1 = f1 X_j (+ g1 S1 + h1 S2), c2 likewise;
    // X_j kept in S1 or S2 for the a kx^2 basis
    int c1 = 0, c2 = -1, keep = 0;
    float f1 = 1.0f, g1 = 0.0f, h1 = 0.0f, f2 = 0.0f, g2 = 0.0f, h2 = 0.0f;
    bool nyq2 = false;
    if (j == kBW3) {
      c1 = L::ETA;
    } else if (j == kBW2) {
      c1 = L::N2;
      keep = TENSOR ? 1 : 0;
    } else if (j == kBVX) {
      c1 = L::V1;
    } else if (j == kBV) {
      c1 = L::V1 + 1, f1 = ck.vy;
      c2 = L::V1 + 2, f2 = ck.vz;
    } else if (j == kBTX) {
      c1 = L::T + 1, f1 = ck.ky;
      c2 = L::T + 2, f2 = ck.kz;
      nyq2 = ck.special;
    } else if (j == kBTA) {
      c1 = L::T + 4, f1 = ck.yz;
      keep = 2;
    } else {  // kBTXX: T_xx and T_yy
      c1 = L::T + 0, f1 = 2.0f * third, g1 = third, h1 = -(ck.ky * ck.ky + ck.kz * ck.kz) * third;
      c2 = L::T + 3, f2 = -third, g2 = third, h2 = (2.0f * ck.ky * ck.ky - ck.kz * ck.kz) * third;
    }
    const bool mix = j == kBTXX;
    col1_inverse_emit<NX, TQ>(bv, q, k1, Eb + buf * TILE, tx, [&](const auto& a, int n1_0, int dn1, int n2) {
      constexpr int K = std::extent_v<std::remove_reference_t<decltype(a)>>;
      if (!col.valid) return;
      cpx* o1 = out + (long long)c1 * Nk + (long long)n2 * plane;
      cpx* o2 = out + (long long)(c2 < 0 ? 0 : c2) * Nk + (long long)n2 * plane;
      if (mix) {  // (uniform per basis: the a kx^2 basis alone reads the kept transforms)
#pragma unroll
        for (int i = 0; i < K; ++i) {
          const int n1 = n1_0 + i * dn1;
          const int x = BX * n1 + n2;
          const long long off = (long long)(BX * n1) * plane;
          cpx v1 = scale(a[i], f1), v2 = scale(a[i], f2);
          const cpx s1 = S1[x * TQ + q], s2 = S2[x * TQ + q];
          v1 = v1 + scale(s1, g1) + scale(s2, h1);
          v2 = v2 + scale(s1, g2) + scale(s2, h2);
          o1[off] = v1;
          o2[off] = v2;
        }
        return;
      }
      if (c2 >= 0) {  // (uniform per basis) two channels, no kept transform
        const cpx c = scale(s_nyq[q], f2);
#pragma unroll
        for (int i = 0; i < K; ++i) {
          const int n1 = n1_0 + i * dn1;
          const int x = BX * n1 + n2;
          const long long off = (long long)(BX * n1) * plane;
          cpx v1 = scale(a[i], f1), v2 = scale(a[i], f2);
          if (nyq2) v2 = (x & 1) ? cpx{-c.x, -c.y} : c;
          o1[off] = v1;
          o2[off] = v2;
        }
        return;
      }
      // one channel, and the transform kept in S1 or S2 for the a kx^2 basis
      cpx* S = keep == 1 ? S1 : S2;
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const int n1 = n1_0 + i * dn1;
        const int x = BX * n1 + n2;
        const long long off = (long long)(BX * n1) * plane;
        o1[off] = scale(a[i], f1);
        if (keep) S[x * TQ + q] = a[i];
      }
    });
    buf ^= 1;
  }
  // mean-field channels: w(k) rho_k with the real weight from the table
  cpx* mf_out = q_out + (long long)b * p.n_chan * Nk;
  for (int m = 0; m < p.M; ++m) {
    cpx bv[BX];
#pragma unroll
    for (int k2 = 0; k2 < BX; ++k2) {
      const long long kidx = (long long)(k1 + AX * k2) * plane + q0 + q;
      const float w = col.valid ? wtab[(5LL + m) * Nk + kidx] : 0.0f;
      bv[k2] = scale(r[k2], w);
    }
    col1_inverse<NX, TQ>(bv, q, k1, Eb + buf * TILE, tx, mf_out + (long long)p.mf_chan_j[m] * Nk, plane, q0);
    buf ^= 1;
  }
}

// Per-thread asynchronous 8-byte copies global -> shared (cp.async, the
// LSU's path; no TMA), committed and waited for in groups.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Backward column pass: F = sum_c conj(W_c) D_c per element (the
// back-convolution), with the bases above.  Each natural-order task
// combines the derivative channels of its column with the column
// constants before one forward x transform per basis:
//   w3: D_eta            i fv kx o_x: D_vx      i fv: ky o_y D_vy + kz o_z D_vz
//   w2: D_n2 + (D_xx + D_yy) / 3                a kx^2: (2 D_xx - D_yy) / 3
//   a: ky^2 D_yy + ky kz c_yz D_yz - (ky^2 + kz^2) / 3 (D_xx + D_yy)
//   a kx c_xy: ky D_xy + kz D_xz (special columns: ky D_xy, and the D_xz
//   term a kx kz sum_x (-1)^x D_xz at the x Nyquist element alone).
// The channel columns stream into four load buffers with cp.async; every
// thread reads back only what it copied itself, and refills a buffer after
// the barrier that follows its last read of it.
template <int NX, int TQ, bool TENSOR>
__global__ void __launch_bounds__(RCol1<NX, TQ>::NT, 2)
    k_rcol_bwd1(EvalParams p, const cpx* __restrict__ pd, const float* __restrict__ wtab, cpx* __restrict__ pf,
                FftTables T) {
  pdl_trigger();
  pdl_wait();
  using L = Lay<false, TENSOR>;
  using C = RCol1<NX, TQ>;
  constexpr int AX = C::AX, BX = C::BX, NT = C::NT, TILE = C::TILE, NF = L::NFMT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx* tx = reinterpret_cast<cpx*>(smem_raw);
  cpx* Eb = tx + NX;
  cpx* Lt = Eb + 2 * TILE;
  __shared__ cpx s_alt[BX * TQ];  // partial sums (-1)^x D_xz of each natural-order task
  const long long plane = (long long)p.ny * p.nzh, Nk = p.Nk;
  const int b = blockIdx.y;
  const long long q0 = (long long)blockIdx.x * TQ;
  const int t = threadIdx.x;
  const int q = t % TQ, k1 = t / TQ;
  const bool nat = t < TQ * BX;
  const int n2 = t / TQ;
  const RColumn col = rk_column(p, q0 + q, (float)p.dky, (float)p.dkz);
  const RColK ck = rk_colk(col);
  const bool ok = col.valid;
  const cpx* src = pd + (long long)b * NF * Nk + q0 + q;
  // this task's samples of channel ch -> load buffer l
  auto load = [&](int ch, int l) {
    if (nat && ok) {
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) {
        const int x = BX * n1 + n2;
        cp_async8(Lt + l * TILE + x * TQ + q, src + (long long)ch * Nk + (long long)x * plane);
      }
    }
  };
  auto at = [&](int l, int n1) { return ok ? Lt[l * TILE + (BX * n1 + n2) * TQ + q] : cpx{0.0f, 0.0f}; };
  if constexpr (TENSOR) {
    load(L::N2, 0);
    load(L::T + 0, 1);
    load(L::T + 3, 2);
    load(L::T + 4, 3);
    cp_async_commit();
  } else {
    load(L::V1 + 1, 0);
    load(L::V1 + 2, 1);
    cp_async_commit();
    load(L::V1, 2);
    cp_async_commit();
    load(L::N2, 3);
    cp_async_commit();
  }
  for (int i = t; i < NX; i += NT) tx[i] = T.tx[i];
  const RTab<BX> tab = rk_task_table<NX, TQ>(wtab, Nk, plane, q0 + q, k1, col.valid);
  const float dkx = (float)p.dkx;
  __syncthreads();
  cpx f[BX];
#pragma unroll
  for (int k2 = 0; k2 < BX; ++k2) f[k2] = cpx{0.0f, 0.0f};
  int buf = 0;
  // One basis: input(a) builds the natural-order samples (natural-order
  // threads), after the barrier refill() issues the next loads, and every
  // spectrum task accumulates conj(W) times the transform.
  auto basis = [&](int j, auto&& input, auto&& refill) {
    cpx* E = Eb + buf * TILE;
    if (nat) {
      cpx a[AX];
      input(a);
      fft::nat_in<NX, false>(a, n2, tx);
#pragma unroll
      for (int kk = 0; kk < AX; ++kk) E[(n2 * AX + kk) * TQ + q] = a[kk];
    }
    __syncthreads();
    refill();
    cpx d[BX];
#pragma unroll
    for (int jj = 0; jj < BX; ++jj) d[jj] = E[(jj * AX + k1) * TQ + q];
    fft::nat_out<NX, false>(d);
    float w[BX];
    const bool odd = rk_basis_weights<NX, TQ>(j, tab, p, k1, dkx, col, w);
    // conj(i w) D = -i w D for an odd basis
#pragma unroll
    for (int k2 = 0; k2 < BX; ++k2)
      f[k2] = odd ? cpx{f[k2].x + w[k2] * d[k2].y, f[k2].y - w[k2] * d[k2].x} : f[k2] + scale(d[k2], w[k2]);
    buf ^= 1;
  };
  auto none = [] {};
  if constexpr (TENSOR) {
    // buffers: 0 n2, 1 xx, 2 yy, 3 yz
    basis(kBTA, [&](cpx (&a)[AX]) {
      cp_async_wait<0>();
      const float c3 = (ck.ky * ck.ky + ck.kz * ck.kz) * (1.0f / 3.0f), cyy = ck.ky * ck.ky - c3;
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = scale(at(2, n1), cyy) + scale(at(3, n1), ck.yz) - scale(at(1, n1), c3);
    }, [&] {
      load(L::T + 1, 3);  // xy -> 3
      cp_async_commit();
    });
    basis(kBW2, [&](cpx (&a)[AX]) {
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = at(0, n1) + scale(at(1, n1) + at(2, n1), 1.0f / 3.0f);
    }, [&] {
      load(L::T + 2, 0);  // xz -> 0
      cp_async_commit();
    });
    basis(kBTXX, [&](cpx (&a)[AX]) {
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = scale(scale(at(1, n1), 2.0f) - at(2, n1), 1.0f / 3.0f);
    }, [&] {
      load(L::V1 + 1, 1);  // vy -> 1, vz -> 2
      load(L::V1 + 2, 2);
      cp_async_commit();
    });
    basis(kBTX, [&](cpx (&a)[AX]) {
      cp_async_wait<1>();  // xy, xz
      const float kz = ck.special ? 0.0f : ck.kz;
      cpx alt{0.0f, 0.0f};
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) {
        const cpx xz = at(0, n1);
        a[n1] = scale(at(3, n1), ck.ky) + scale(xz, kz);
        alt = ((BX * n1 + n2) & 1) ? alt - xz : alt + xz;
      }
      s_alt[n2 * TQ + q] = alt;
    }, [&] {
      load(L::V1, 3);  // vx -> 3
      cp_async_commit();
      load(L::ETA, 0);  // eta -> 0
      cp_async_commit();
      // the D_xz term of a special column at the x Nyquist element
      if (ck.special && k1 == C::K1N) {
        cpx s{0.0f, 0.0f};
#pragma unroll
        for (int jj = 0; jj < BX; ++jj) s = s + s_alt[jj * TQ + q];
        f[C::K2N] = f[C::K2N] + scale(s, tab.a[C::K2N] * (dkx * (float)C::KN) * ck.kz);
      }
    });
    basis(kBV, [&](cpx (&a)[AX]) {
      cp_async_wait<2>();  // vy, vz
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = scale(at(1, n1), ck.vy) + scale(at(2, n1), ck.vz);
    }, none);
    basis(kBVX, [&](cpx (&a)[AX]) {
      cp_async_wait<1>();
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = at(3, n1);
    }, none);
    basis(kBW3, [&](cpx (&a)[AX]) {
      cp_async_wait<0>();
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = at(0, n1);
    }, none);
  } else {
    // buffers: 0 vy, 1 vz, 2 vx, 3 n2
    basis(kBV, [&](cpx (&a)[AX]) {
      cp_async_wait<2>();
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = scale(at(0, n1), ck.vy) + scale(at(1, n1), ck.vz);
    }, [&] {
      load(L::ETA, 0);  // eta -> 0
      cp_async_commit();
    });
    basis(kBVX, [&](cpx (&a)[AX]) {
      cp_async_wait<2>();
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = at(2, n1);
    }, none);
    basis(kBW2, [&](cpx (&a)[AX]) {
      cp_async_wait<1>();
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = at(3, n1);
    }, none);
    basis(kBW3, [&](cpx (&a)[AX]) {
      cp_async_wait<0>();
#pragma unroll
      for (int n1 = 0; n1 < AX; ++n1) a[n1] = at(0, n1);
    }, none);
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  col1_inverse<NX, TQ>(f, q, k1, Eb + buf * TILE, tx, pf + (long long)b * Nk, plane, q0);
}

}  // namespace rk
}  // namespace cdft
