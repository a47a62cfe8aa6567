// Launchers of the fused transform path (fused.cu, kernels in
// fft_reg_kernels.cuh).  Specialisations exist for nx in {16, 32, 48, 64, 96,
// 128} and (ny, nz) in the same set squared; fused_plan reports whether an
// engine's grid and channel count have one.
#pragma once

#include "cdft_common.cuh"
#include "fft_core.cuh"

namespace cdft {

struct FusedPlan {
  size_t plane_smem = 0, colf_smem = 0, colb_smem = 0;
  int tq = 0;         // columns per column-pass tile
  int col_tiles = 0;  // column-pass CTAs per problem
  bool tq32 = false;  // several species: 32-column tiles fit (16 always do)
  // the two middle plane passes (channels inverse, derivatives forward) with
  // twice the threads per plane CTA (RPlane::NT_WIDE instead of NT)
  bool plane_wide = false;
  // programmatic dependent launch of the passes whose stream predecessor is
  // the previous pass (set per evaluation: off while timing stages)
  bool pdl = false;
};

// Column tile width of the plan (16, or 32 where tq32): false, plan
// unchanged, for a width it does not have.
bool fused_plan_set_tile(const EvalParams& p, FusedPlan* plan, int tq);

// True (and `plan` filled, the kernels' shared-memory limits raised) when the
// fused path serves this engine.
bool fused_plan(const EvalParams& p, FusedPlan* plan);

// err: the engine's error word, set when a bounded wait of a bulk copy
// gives up (cdft_engine_status reports it).
// The rho plane pass writes each plane's mean (pmean, B * S * nx doubles);
// the column pass turns them into the species means (mean, B * kMaxSpecies)
// of the mixed-precision split.
void fused_plane_fwd_rho(const FusedPlan& f, const EvalParams& p, const double* rho, double* pmean,
                         fft::cpx* prho, int* err, const FftTables& T, cudaStream_t st);
// The column pass reads the FMT and mean-field weights from a table built
// once per engine (after the mean-field weights).
long long fused_weight_table_floats(const EvalParams& p);
void fused_build_weights(const EvalParams& p, const double* mf_w, float* wtab, cudaStream_t st);

void fused_col_fwd(const FusedPlan& f, const EvalParams& p, const fft::cpx* prho, const double* pmean, double* mean,
                   const float* wtab, fft::cpx* q, const FftTables& T, cudaStream_t st);
// The two middle plane passes take x planes ix0 .. ix0 + nplanes - 1 (the
// engine may split them into concurrent chunks).
void fused_plane_inv(const FusedPlan& f, const EvalParams& p, const fft::cpx* q, float* chan_r, int* err, int ix0,
                     int nplanes, const FftTables& T, cudaStream_t st);
void fused_plane_fwd_deriv(const FusedPlan& f, const EvalParams& p, const float* deriv_r, fft::cpx* pd, int* err,
                           int ix0, int nplanes, const FftTables& T, cudaStream_t st);
void fused_col_bwd(const FusedPlan& f, const EvalParams& p, const fft::cpx* pd, const float* wtab, fft::cpx* pf,
                   const FftTables& T, cudaStream_t st);
void fused_plane_inv_epi(const FusedPlan& f, const EvalParams& p, const fft::cpx* pf, const double* dbar,
                         double* force, const MuArgs& mu, const FinalArgs& fin, int* err, const FftTables& T,
                         cudaStream_t st);

}  // namespace cdft
