// Instantiations and launchers of the fused transform path (the kernels are
// in fft_kernels.cuh): dispatch from runtime grid sizes and channel layout to
// the size-specialised kernels.
#include "fused.cuh"

#include <type_traits>

#include "fft_kernels.cuh"

namespace cdft {

namespace {

constexpr size_t kSmemCap = 110 * 1024;     // plane kernels: two CTAs per SM at least
constexpr size_t kColSmemCap = 74 * 1024;   // column kernels: three CTAs per SM

template <int N>
using IC = std::integral_constant<int, N>;

// f(IC<n>) for a supported transform length n; false otherwise.
template <class F>
bool with_len(int n, F&& f) {
  switch (n) {
    case 16: f(IC<16>{}); return true;
    case 32: f(IC<32>{}); return true;
    case 64: f(IC<64>{}); return true;
    case 128: f(IC<128>{}); return true;
    default: return false;
  }
}

template <class F>
bool with_plane(int ny, int nz, F&& f) {
  bool ok = false;
  with_len(ny, [&](auto yc) { ok = with_len(nz, [&](auto zc) { f(yc, zc); }); });
  return ok;
}

template <class F>
void with_layout(const EvalParams& p, F&& f) {
  if (p.L.multi) {
    if (p.L.tensor)
      f(std::true_type{}, std::true_type{});
    else
      f(std::true_type{}, std::false_type{});
  } else {
    if (p.L.tensor)
      f(std::false_type{}, std::true_type{});
    else
      f(std::false_type{}, std::false_type{});
  }
}

template <class K>
void allow_smem(K kern, size_t bytes) {
  CDFT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

}  // namespace

bool fused_plan(const EvalParams& p, FusedPlan* plan) {
  FusedPlan f;
  bool ok = with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    constexpr int NY = decltype(yc)::value, NZ = decltype(zc)::value;
    f.plane_smem = Plane<NY, NZ, kPlaneThreads>::kSmem;
  });
  ok = ok && with_len(p.nx, [](auto) {});
  if (!ok || f.plane_smem > kSmemCap) return false;
  // column tiles: the widest (at most 16 columns) whose buffers leave room
  // for three CTAs per SM (one CTA's worth of buffers at the least)
  f.ltq = 4;
  while (f.ltq > 0 &&
         (col_smem(p.nx, f.ltq, p.S + p.n_chan) > kColSmemCap || col_smem(p.nx, f.ltq, p.L.n_deriv) > kColSmemCap))
    --f.ltq;
  f.colf_smem = col_smem(p.nx, f.ltq, p.S + p.n_chan);
  f.colb_smem = col_smem(p.nx, f.ltq, p.L.n_deriv);
  if (f.colf_smem > kSmemCap || f.colb_smem > kSmemCap) return false;
  f.col_tiles = (int)(((long long)p.ny * p.nzh + (1 << f.ltq) - 1) >> f.ltq);
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    constexpr int NY = decltype(yc)::value, NZ = decltype(zc)::value;
    allow_smem(k_plane_fwd<NY, NZ, double, kPlaneThreadsWide>, f.plane_smem);
    allow_smem(k_plane_fwd<NY, NZ, float, kPlaneThreads>, f.plane_smem);
    allow_smem(k_plane_inv<NY, NZ>, f.plane_smem);
    with_layout(p, [&](auto mc, auto tc) {
      allow_smem(k_plane_inv_epi<NY, NZ, decltype(mc)::value, decltype(tc)::value>, f.plane_smem);
    });
  });
  with_len(p.nx, [&](auto xc) {
    constexpr int NX = decltype(xc)::value;
    with_layout(p, [&](auto mc, auto tc) {
      constexpr bool MU = decltype(mc)::value, TE = decltype(tc)::value;
      allow_smem(k_col_fwd<NX, MU, TE>, f.colf_smem);
      allow_smem(k_col_bwd<NX, MU, TE>, f.colb_smem);
    });
  });
  *plan = f;
  return true;
}

void fused_plane_fwd_rho(const FusedPlan& f, const EvalParams& p, const double* rho, const double* mean,
                         fft::cpx* prho, const FftTables& T, cudaStream_t st) {
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    k_plane_fwd<decltype(yc)::value, decltype(zc)::value, double, kPlaneThreadsWide>
        <<<dim3(p.nx, p.S, p.batch), kPlaneThreadsWide, f.plane_smem, st>>>(p, rho, p.S, mean, prho, T);
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_col_fwd(const FusedPlan& f, const EvalParams& p, const fft::cpx* prho, const double* mf_w,
                   const float* wtab, fft::cpx* q, const FftTables& T, cudaStream_t st) {
  with_len(p.nx, [&](auto xc) {
    with_layout(p, [&](auto mc, auto tc) {
      k_col_fwd<decltype(xc)::value, decltype(mc)::value, decltype(tc)::value>
          <<<dim3(f.col_tiles, p.batch), kColThreads, f.colf_smem, st>>>(p, prho, mf_w, wtab, q, f.ltq, T);
    });
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_plane_inv(const FusedPlan& f, const EvalParams& p, const fft::cpx* q, float* chan_r, const FftTables& T,
                     cudaStream_t st) {
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    k_plane_inv<decltype(yc)::value, decltype(zc)::value>
        <<<dim3(p.nx, p.n_chan, p.batch), kPlaneThreads, f.plane_smem, st>>>(p, q, p.n_chan, chan_r, T);
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_plane_fwd_deriv(const FusedPlan& f, const EvalParams& p, const float* deriv_r, fft::cpx* pd,
                           const FftTables& T, cudaStream_t st) {
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    k_plane_fwd<decltype(yc)::value, decltype(zc)::value, float, kPlaneThreads>
        <<<dim3(p.nx, p.L.n_deriv, p.batch), kPlaneThreads, f.plane_smem, st>>>(p, deriv_r, p.L.n_deriv, nullptr,
                                                                                 pd, T);
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_col_bwd(const FusedPlan& f, const EvalParams& p, const fft::cpx* pd, const float* wtab, fft::cpx* pf,
                   const FftTables& T, cudaStream_t st) {
  with_len(p.nx, [&](auto xc) {
    with_layout(p, [&](auto mc, auto tc) {
      k_col_bwd<decltype(xc)::value, decltype(mc)::value, decltype(tc)::value>
          <<<dim3(f.col_tiles, p.batch), kColThreads, f.colb_smem, st>>>(p, pd, wtab, pf, f.ltq, T);
    });
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_plane_inv_epi(const FusedPlan& f, const EvalParams& p, const fft::cpx* pf, const double* dbar,
                         double* force, const MuArgs& mu, const FinalArgs& fin, const FftTables& T, cudaStream_t st) {
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    with_layout(p, [&](auto mc, auto tc) {
      k_plane_inv_epi<decltype(yc)::value, decltype(zc)::value, decltype(mc)::value, decltype(tc)::value>
          <<<dim3(p.nx, p.S, p.batch), kPlaneThreadsWide, f.plane_smem, st>>>(p, pf, dbar, force, mu, fin, T);
    });
  });
  CDFT_CUDA(cudaGetLastError());
}

long long fused_weight_table_floats(const EvalParams& p) { return weight_table_floats(p); }

void fused_build_weights(const EvalParams& p, float* wtab, cudaStream_t st) {
  k_build_weights<<<592, 256, 0, st>>>(p, wtab);
  CDFT_CUDA(cudaGetLastError());
}

}  // namespace cdft
