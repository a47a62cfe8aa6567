// The ideal-gas and external-field terms of the functional without any device
// allocation (ideal_gas.hpp:18-37, external_field.hpp:16-30): a variant of the
// local-term part of the pointwise kernel whose reduction scratch is a
// file-scope device array instead of engine memory.
//
// Who needs this: callers that cannot call cudaMalloc (or anything that
// allocates) at the point where they evaluate -- code running under a custom
// or pool allocator that forbids foreign allocations, host code that must not
// allocate while another library holds the device, or any caller that owns
// all of its device memory up front.  They pass their own input and output
// buffers; the only scratch is the array below.
//
// The array is part of the library image: every GPU that loads the library
// holds its 28 KiB until the process exits.  All calls share it, so two calls
// whose kernels overlap on the GPU (different streams, or different host
// threads on one device) race on it: serialise them.  The partial sums are
// fully rewritten by every call before they are read, so nothing carries over
// from the previous call.
#include <string>

#include "../../include/cdft_b200.h"
#include "cdft_common.cuh"

namespace {

constexpr int kNaBlocks = 592;                        // 4 CTAs per SM on 148 SMs
constexpr int kNaTerms = 2 + cdft::kMaxSpecies;       // F_id, F_ext, N_0..N_3
constexpr int kNaThreads = 256;

// kNaBlocks x kNaTerms partial sums: 592 * 6 * 8 bytes = 28 KiB.
static __device__ __align__(256) double g_noalloc_scratch[kNaBlocks * kNaTerms];

struct NaArgs {
  const double* rho;
  const double* vext;
  double mu[cdft::kMaxSpecies];
  int S;
  long long N;
  double dv;
  double* force;
};

// Local force (ln rho - mu + V) dV per point and per-block partial sums of
// rho (ln rho - 1), rho V and rho.
__global__ void __launch_bounds__(kNaThreads) k_local_terms(NaArgs a, double* __restrict__ partials) {
  double acc[kNaTerms];
#pragma unroll
  for (int t = 0; t < kNaTerms; ++t) acc[t] = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x)
#pragma unroll
    for (int s = 0; s < cdft::kMaxSpecies; ++s) {
      if (s < a.S) {
        const double r = a.rho[s * a.N + i];
        const double v = a.vext ? a.vext[s * a.N + i] : 0.0;
        const double lr = log(r < 1e-300 ? 1e-300 : r);
        acc[0] += r * (lr - 1.0);
        acc[1] += r * v;
        acc[2 + s] += r;
        a.force[s * a.N + i] = (lr - a.mu[s]) * a.dv + v * a.dv;
      }
    }
  __shared__ double sh[kNaThreads / 32][kNaTerms];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < kNaTerms; ++t) {
    double v = acc[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp][t] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNaTerms) {
    double v = 0.0;
    for (int w = 0; w < kNaThreads / 32; ++w) v += sh[w][threadIdx.x];
    partials[blockIdx.x * kNaTerms + threadIdx.x] = v;
  }
}

// [F_id, F_ext, N_0 .. N_{S-1}] = dV * (sum over the blocks), one warp per term.
__global__ void k_local_finish(const double* __restrict__ partials, int nblocks, int S, double dv,
                               double* __restrict__ out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp >= 2 + S) return;
  double v = 0.0;
  for (int b = lane; b < nblocks; b += 32) v += partials[b * kNaTerms + warp];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) out[warp] = v * dv;
}

// With the caller's device current: the device address of the scratch
// array.  In host code `g_noalloc_scratch` names a host-side stand-in, not
// device memory, so it is never passed to a kernel directly.  The address is
// looked up on every call rather than cached: a device reset or a new primary
// context reloads the module, and the array may then sit elsewhere.
double* scratch_for_current_device(std::string& err) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    err = std::string("cudaGetDevice failed: ") + cudaGetErrorString(e);
    return nullptr;
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    err = std::string("cudaGetSymbolAddress failed on device ") + std::to_string(dev) + ": " +
          cudaGetErrorString(e);
    return nullptr;
  }
  return static_cast<double*>(p);
}

}  // namespace

namespace cdft {
// The C ABI's thread-local error message (capi.cu).
void set_last_error(const std::string& msg);
}  // namespace cdft

extern "C" int cdft_local_terms_noalloc(const double* rho, const double* vext, const double* mu, int n_species,
                                        long long n_points, double dv, double* force, double* scalars,
                                        void* stream) {
  if (!rho || !mu || !force || !scalars) {
    cdft::set_last_error("cdft_local_terms_noalloc: rho, mu, force and scalars are required");
    return CDFT_ERR_INVALID;
  }
  if (n_species < 1 || n_species > cdft::kMaxSpecies) {
    cdft::set_last_error("cdft_local_terms_noalloc: n_species must be in [1, 4] (the scratch array holds " +
                         std::to_string(kNaBlocks) + " x " + std::to_string(kNaTerms) + " partial sums)");
    return CDFT_ERR_INVALID;
  }
  if (n_points < 1 || !(dv > 0.0)) {
    cdft::set_last_error("cdft_local_terms_noalloc: n_points must be >= 1 and dv > 0");
    return CDFT_ERR_INVALID;
  }
  std::string err;
  double* scratch = scratch_for_current_device(err);
  if (!scratch) {
    cdft::set_last_error("cdft_local_terms_noalloc: " + err);
    return CDFT_ERR_CUDA;
  }
  NaArgs a;
  a.rho = rho;
  a.vext = vext;
  for (int s = 0; s < cdft::kMaxSpecies; ++s) a.mu[s] = s < n_species ? mu[s] : 0.0;
  a.S = n_species;
  a.N = n_points;
  a.dv = dv;
  a.force = force;
  const long long want = (n_points + kNaThreads - 1) / kNaThreads;
  const int blocks = (int)(want < kNaBlocks ? want : kNaBlocks);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_local_terms<<<blocks, kNaThreads, 0, st>>>(a, scratch);
  k_local_finish<<<1, 32 * kNaTerms, 0, st>>>(scratch, blocks, n_species, dv, scalars);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cdft::set_last_error(std::string("cdft_local_terms_noalloc: launch failed: ") + cudaGetErrorString(e));
    return CDFT_ERR_CUDA;
  }
  return CDFT_OK;
}
