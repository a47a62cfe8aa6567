// Instantiations and launchers of the fused transform path (the kernels are
// in fft_reg_kernels.cuh): dispatch from runtime grid sizes and channel
// layout to the size-specialised kernels.
#include "fused.cuh"

#include <type_traits>

#include "fft_reg_kernels.cuh"

namespace cdft {

namespace {

constexpr size_t kSmemCap = 110 * 1024;  // two CTAs per SM at least

template <int N>
using IC = std::integral_constant<int, N>;

// f(IC<n>) for a supported transform length n; false otherwise.
template <class F>
bool with_len(int n, F&& f) {
  switch (n) {
    case 16: f(IC<16>{}); return true;
    case 32: f(IC<32>{}); return true;
    case 48: f(IC<48>{}); return true;
    case 64: f(IC<64>{}); return true;
    case 96: f(IC<96>{}); return true;
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

// f(IC<tq>) for the column tile width of the plan.
template <class F>
void with_tq(int tq, F&& f) {
  if (tq == 32)
    f(IC<32>{});
  else
    f(IC<16>{});
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
    f.plane_smem = rk::RPlane<NY, NZ>::kSmem;
  });
  ok = ok && with_len(p.nx, [](auto) {});
  if (!ok || f.plane_smem > kSmemCap) return false;
  // column tiles: one species keeps its spectra in registers (16 columns
  // a tile); several keep them in shared memory (32 columns unless their
  // spectra need narrower tiles)
  if (p.S == 1) {
    f.tq = 16;
    f.colf_smem = rk::rcol1_smem(p.nx, f.tq);
    f.colb_smem = rk::rcol1_smem_bwd(p.nx, f.tq);
  } else {
    f.tq32 = rk::rcol_smem(p.nx, 32, p.S) <= kSmemCap;
    f.tq = f.tq32 ? 32 : 16;
    f.colf_smem = rk::rcol_smem(p.nx, f.tq, p.S);
    f.colb_smem = f.colf_smem;
  }
  if (f.colf_smem > kSmemCap || f.colb_smem > kSmemCap) return false;
  f.col_tiles = (int)(((long long)p.ny * p.nzh + f.tq - 1) / f.tq);
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    constexpr int NY = decltype(yc)::value, NZ = decltype(zc)::value;
    allow_smem(rk::k_rplane_fwd<NY, NZ, double, rk::RPlane<NY, NZ>::NT_WIDE>, f.plane_smem);
    constexpr int NTW = rk::RPlane<NY, NZ>::NT_WIDE;
    allow_smem(rk::k_rplane_fwd<NY, NZ, float>, f.plane_smem);
    allow_smem(rk::k_rplane_fwd<NY, NZ, float, NTW>, f.plane_smem);
    with_layout(p, [&](auto mc, auto tc) {
      constexpr bool MU = decltype(mc)::value, TE = decltype(tc)::value;
      allow_smem(rk::k_rplane_inv<NY, NZ, false, MU, TE>, f.plane_smem);
      allow_smem(rk::k_rplane_inv<NY, NZ, false, MU, TE, NTW>, f.plane_smem);
      allow_smem(rk::k_rplane_inv<NY, NZ, true, MU, TE, NTW>, f.plane_smem);
    });
  });
  with_len(p.nx, [&](auto xc) {
    constexpr int NX = decltype(xc)::value;
    // every tile width the plan may switch to (several species: 16 and,
    // where it fits, 32)
    for (int tq : {16, 32}) {
      if (tq != f.tq && !(p.S > 1 && tq == 16) && !(tq == 32 && f.tq32)) continue;
      const size_t sm = p.S > 1 ? rk::rcol_smem(p.nx, tq, p.S) : 0;
      with_tq(tq, [&](auto qc) {
        constexpr int TQ = decltype(qc)::value;
        with_layout(p, [&](auto mc, auto tc) {
          constexpr bool MU = decltype(mc)::value, TE = decltype(tc)::value;
          if constexpr (MU) {
            allow_smem(rk::k_rcol_fwd<NX, TQ, MU, TE>, sm);
            allow_smem(rk::k_rcol_bwd<NX, TQ, MU, TE>, sm);
          } else if constexpr (TQ == 16) {  // one species: 16-column tiles only
            allow_smem(rk::k_rcol_fwd1<NX, TQ, TE>, f.colf_smem);
            allow_smem(rk::k_rcol_bwd1<NX, TQ, TE>, f.colb_smem);
          }
        });
      });
    }
  });
  *plan = f;
  return true;
}

bool fused_plan_set_tile(const EvalParams& p, FusedPlan* f, int tq) {
  if (p.S == 1) return tq == 16;  // one species: 16-column tiles only
  if (tq != 16 && !(tq == 32 && f->tq32)) return false;
  f->tq = tq;
  f->colf_smem = rk::rcol_smem(p.nx, tq, p.S);
  f->colb_smem = f->colf_smem;
  f->col_tiles = (int)(((long long)p.ny * p.nzh + tq - 1) / tq);
  return true;
}

void fused_plane_fwd_rho(const FusedPlan& f, const EvalParams& p, const double* rho, double* pmean,
                         fft::cpx* prho, int* err, const FftTables& T, cudaStream_t st) {
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    constexpr int NY = decltype(yc)::value, NZ = decltype(zc)::value;
    constexpr int NT = rk::RPlane<NY, NZ>::NT_WIDE;
    rk::k_rplane_fwd<NY, NZ, double, NT>
        <<<dim3(p.nx, p.S, p.batch), NT, f.plane_smem, st>>>(p, rho, p.S, pmean, prho, err, 0, T);
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_col_fwd(const FusedPlan& f, const EvalParams& p, const fft::cpx* prho, const double* pmean, double* mean,
                   const float* wtab, fft::cpx* q, const FftTables& T, cudaStream_t st) {
  with_len(p.nx, [&](auto xc) {
    with_tq(f.tq, [&](auto qc) {
      with_layout(p, [&](auto mc, auto tc) {
        constexpr int NX = decltype(xc)::value, TQ = decltype(qc)::value;
        constexpr bool MU = decltype(mc)::value, TE = decltype(tc)::value;
        // (stream predecessor: the rho plane pass)
        if constexpr (MU)
          launch_k(rk::k_rcol_fwd<NX, TQ, MU, TE>, dim3(f.col_tiles, p.batch), dim3(rk::RCol<NX>::NT), f.colf_smem,
                   st, f.pdl, p, prho, pmean, mean, wtab, q, T);
        else if constexpr (TQ == 16)
          launch_k(rk::k_rcol_fwd1<NX, TQ, TE>, dim3(f.col_tiles, p.batch), dim3(rk::RCol1<NX, TQ>::NT),
                   f.colf_smem, st, f.pdl, p, prho, pmean, mean, wtab, q, T);
      });
    });
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_plane_inv(const FusedPlan& f, const EvalParams& p, const fft::cpx* q, float* chan_r, int* err, int ix0,
                     int nplanes, const FftTables& T, cudaStream_t st) {
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    constexpr int NY = decltype(yc)::value, NZ = decltype(zc)::value;
    with_layout(p, [&](auto mc, auto tc) {
      constexpr bool MU = decltype(mc)::value, TE = decltype(tc)::value;
      auto go = [&](auto nc) {
        constexpr int NT = decltype(nc)::value;
        rk::k_rplane_inv<NY, NZ, false, MU, TE, NT><<<dim3(nplanes, p.n_chan, p.batch), NT, f.plane_smem, st>>>(
            p, q, p.n_chan, chan_r, nullptr, nullptr, MuArgs{}, FinalArgs{nullptr, 0, nullptr, nullptr}, err, ix0, T);
      };
      if (f.plane_wide)
        go(IC<rk::RPlane<NY, NZ>::NT_WIDE>{});
      else
        go(IC<rk::RPlane<NY, NZ>::NT>{});
    });
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_plane_fwd_deriv(const FusedPlan& f, const EvalParams& p, const float* deriv_r, fft::cpx* pd, int* err,
                           int ix0, int nplanes, const FftTables& T, cudaStream_t st) {
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    constexpr int NY = decltype(yc)::value, NZ = decltype(zc)::value;
    // (stream predecessor: the chunk's pointwise kernel)
    auto go = [&](auto nc) {
      constexpr int NT = decltype(nc)::value;
      launch_k(rk::k_rplane_fwd<NY, NZ, float, NT>, dim3(nplanes, p.L.n_deriv, p.batch), dim3(NT), f.plane_smem, st,
               f.pdl, p, deriv_r, p.L.n_deriv, (double*)nullptr, pd, err, ix0, T);
    };
    if (f.plane_wide)
      go(IC<rk::RPlane<NY, NZ>::NT_WIDE>{});
    else
      go(IC<rk::RPlane<NY, NZ>::NT>{});
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_col_bwd(const FusedPlan& f, const EvalParams& p, const fft::cpx* pd, const float* wtab, fft::cpx* pf,
                   const FftTables& T, cudaStream_t st) {
  with_len(p.nx, [&](auto xc) {
    with_tq(f.tq, [&](auto qc) {
      with_layout(p, [&](auto mc, auto tc) {
        constexpr int NX = decltype(xc)::value, TQ = decltype(qc)::value;
        constexpr bool MU = decltype(mc)::value, TE = decltype(tc)::value;
        if constexpr (MU)
          rk::k_rcol_bwd<NX, TQ, MU, TE>
              <<<dim3(f.col_tiles, p.batch), rk::RCol<NX>::NT, f.colb_smem, st>>>(p, pd, wtab, pf, T);
        else if constexpr (TQ == 16)
          rk::k_rcol_bwd1<NX, TQ, TE>
              <<<dim3(f.col_tiles, p.batch), rk::RCol1<NX, TQ>::NT, f.colb_smem, st>>>(p, pd, wtab, pf, T);
      });
    });
  });
  CDFT_CUDA(cudaGetLastError());
}

void fused_plane_inv_epi(const FusedPlan& f, const EvalParams& p, const fft::cpx* pf, const double* dbar,
                         double* force, const MuArgs& mu, const FinalArgs& fin, int* err, const FftTables& T,
                         cudaStream_t st) {
  with_plane(p.ny, p.nz, [&](auto yc, auto zc) {
    constexpr int NY = decltype(yc)::value, NZ = decltype(zc)::value;
    with_layout(p, [&](auto mc, auto tc) {
      constexpr int NT = rk::RPlane<NY, NZ>::NT_WIDE;
      // (stream predecessor: the backward column pass)
      launch_k(rk::k_rplane_inv<NY, NZ, true, decltype(mc)::value, decltype(tc)::value, NT>, dim3(p.nx, p.S, p.batch),
               dim3(NT), f.plane_smem, st, f.pdl, p, pf, p.S, (float*)nullptr, force, dbar, mu, fin, err, 0, T);
    });
  });
  CDFT_CUDA(cudaGetLastError());
}

long long fused_weight_table_floats(const EvalParams& p) { return rk::rweight_table_floats(p); }

void fused_build_weights(const EvalParams& p, const double* mf_w, float* wtab, cudaStream_t st) {
  rk::k_build_rweights<<<592, 256, 0, st>>>(p, mf_w, wtab);
  CDFT_CUDA(cudaGetLastError());
}

}  // namespace cdft
