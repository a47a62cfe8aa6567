// Shared definitions of the classicalDFT B200 engine: evaluation parameters,
// channel layouts, complex helpers and error plumbing.
//
// Layouts (identical to the reference, include/dft/grid.hpp:35-63):
//   real field   : N  = nx*ny*nz doubles, flat index iz + nz*(iy + ny*ix)
//   k-space field: Nk = nx*ny*(nz/2+1) complex values, index iz + nzh*(iy + ny*ix)
// Multi-channel arrays are channel-major: channel c occupies [c*N, (c+1)*N)
// (or [c*Nk, (c+1)*Nk) in k-space), so every kernel reads each channel with
// fully coalesced warps and cuFFT runs one batched plan over all channels.
#pragma once

#include <utility>

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace cdft {

constexpr int kMaxSpecies = 4;
constexpr int kMaxInteractions = 8;
// Problems of one shape evaluated together by a batched engine (one set of
// launches; the problem index is blockIdx.y).
constexpr int kMaxBatch = 64;
constexpr double kPi = 3.14159265358979323846;

// FMT model ids (include/dft/functionals/fmt/models.hpp:153-359).
enum ModelId : int { kRosenfeld = 0, kRSLT = 1, kWhiteBearI = 2, kWhiteBearII = 3, kEsFMT = 4 };

__host__ __device__ constexpr bool model_has_tensor(int m) {
  return m == kWhiteBearI || m == kWhiteBearII || m == kEsFMT;
}

// Tensor component order of the six stored channels (weights.hpp:46-50):
// xx, xy, xz, yy, yz, zz.
__host__ __device__ constexpr int tensor_index(int i, int j) {
  return (i > j) ? (j == 0 ? i : (j == 1 ? 2 + i : 5)) : (i == 0 ? j : (i == 1 ? 2 + j : 5));
}

// Forward (weighted-density) channel layout.
//   one species  : eta, n2, v[3], T[5]                  (5 or 10 channels)
//   mixtures     : eta, n2, n1, n0, v1[3], v0[3], T[5]  (10 or 15 channels)
// followed by the mean-field convolution channels.  Only five tensor
// components are transformed (xx, xy, xz, yy, yz): the trace of the tensor
// weight is the surface weight (A + 3B = w2 in weights.hpp:121-137), so
// T_zz = n2 - T_xx - T_yy exactly, and in the back-convolution dPhi/dT_zz
// folds into the n2, xx and yy channels.  The derivative channels use the
// same order; for one species n1/n0 and v0 are folded into n2 and v before
// the transform (hard_sphere.hpp:121,125).
struct ChannelLayout {
  int multi = 0;       // species-summed n1, n0, v0 channels present
  int tensor = 0;      // tensor channels present
  int eta = 0, n2 = 1, n1 = -1, n0 = -1, v1 = 2, v0 = -1, t = 5;
  int n_fmt = 5;       // FMT channels
  int n_deriv = 5;     // derivative channels
  static ChannelLayout make(bool multi, bool tensor) {
    ChannelLayout L;
    L.multi = multi;
    L.tensor = tensor;
    if (!multi) {
      L.eta = 0; L.n2 = 1; L.v1 = 2; L.t = 5;
      L.n_fmt = tensor ? 10 : 5;
    } else {
      L.eta = 0; L.n2 = 1; L.n1 = 2; L.n0 = 3; L.v1 = 4; L.v0 = 7; L.t = 10;
      L.n_fmt = tensor ? 15 : 10;
    }
    L.n_deriv = L.n_fmt;
    return L;
  }
};

constexpr int kMaxChannels = 15 + 2 * kMaxInteractions;

struct EvalParams {
  int nx, ny, nz, nzh;
  long long N, Nk;
  double dx, dv, inv_n;
  double dkx, dky, dkz;
  int S;
  double R[kMaxSpecies];
  double inv4piR[kMaxSpecies];
  double inv4piR2[kMaxSpecies];
  int model;
  double A, B;
  ChannelLayout L;
  int M;                          // mean-field interactions
  int mf_i[kMaxInteractions], mf_j[kMaxInteractions];
  int mf_chan_j[kMaxInteractions];  // channel holding w * rho_j
  int mf_chan_i[kMaxInteractions];  // channel holding w * rho_i (cross terms), else -1
  int n_chan;                       // FMT + mean-field channels
  int n_terms;                      // reduction terms
  int batch;                        // problems evaluated together (1..kMaxBatch)
};

// Chemical potentials (beta mu) of every problem of a batch, passed to the
// kernels that need them as a __grid_constant__ parameter.
struct MuArgs {
  double mu[kMaxBatch][kMaxSpecies];
};

// Inputs of the final reduction folded into k_epilogue (scalars == null
// skips it).
struct FinalArgs {
  const double* partials;  // B * nblocks * n_terms (the pointwise kernel's)
  int nblocks;
  const int* err;
  double* scalars;         // B * kScalarCount
};

// Reduction term order: F_hs, F_id, F_ext, F_mf, then N_s for each species.
enum Term : int { kTermHS = 0, kTermId = 1, kTermExt = 2, kTermMF = 3, kTermN0 = 4 };

// Scalar output order written by the engine (device and host variants):
// F, Omega, F_id, F_ext, F_hs, F_mf, N_0..N_{S-1} (N_s = sum rho_s dV).
constexpr int kScalarCount = 6 + kMaxSpecies;

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }
 private:
  int code_;
};

}  // namespace cdft

#define CDFT_CUDA(call)                                                                     \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::cdft::Error(-3, std::string("CUDA error ") + cudaGetErrorString(e_) + " at " + \
                                  __FILE__ + ":" + std::to_string(__LINE__));               \
  } while (0)

// Programmatic dependent launch.  A kernel launched with the attribute
// (launch_k with pdl) may be scheduled while its stream predecessor still
// runs; pdl_wait() blocks until that predecessor has completed and its
// writes are visible (a no-op in a launch without the attribute).
// pdl_trigger() lets this grid's dependent be scheduled once every CTA of
// this grid has started (so the dependent's waiting CTAs never keep this
// grid's later CTAs from starting).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... Exp, class... Act>
inline void launch_k(void (*kern)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                     Act&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  CDFT_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Act>(args)...));
}

#define CDFT_CUFFT(call)                                                                   \
  do {                                                                                     \
    cufftResult r_ = (call);                                                               \
    if (r_ != CUFFT_SUCCESS)                                                               \
      throw ::cdft::Error(-4, std::string("cuFFT error ") + std::to_string((int)r_) + " at " + \
                                  __FILE__ + ":" + std::to_string(__LINE__));              \
  } while (0)
