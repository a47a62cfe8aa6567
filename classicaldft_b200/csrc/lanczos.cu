// Block Lanczos for the lowest Hessian eigenpair: see lanczos.cuh.
#include "lanczos.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace cdft {

namespace {

constexpr int kT = 256;     // threads of the vector kernels
constexpr int kMaxBlock = 4;

__device__ __forceinline__ bool lz_face(long long i, int nx, int ny, int nz) {
  const int iz = (int)(i % nz);
  const long long t = i / nz;
  const int iy = (int)(t % ny);
  const int ix = (int)(t / ny);
  return ix == 0 || ix == nx - 1 || iy == 0 || iy == ny - 1 || iz == 0 || iz == nz - 1;
}

__device__ __forceinline__ unsigned long long lz_hash(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Seeded standard normal draws on the interior, zero on the faces.
__global__ void k_lz_randn(double* __restrict__ out, long long N, unsigned long long seed, int nx, int ny, int nz) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long a = lz_hash(seed * 0x100000001b3ull + 2 * i);
    const unsigned long long b = lz_hash(seed * 0x100000001b3ull + 2 * i + 1);
    const double u1 = ((a >> 11) + 1.0) * (1.0 / 9007199254740993.0);  // (0, 1]
    const double u2 = (b >> 11) * (1.0 / 9007199254740992.0);
    out[i] = lz_face(i, nx, ny, nz) ? 0.0 : sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
  }
}

// out = in with the faces zeroed (in may equal out); nvec vectors of N.
__global__ void k_lz_faces(const double* in, double* out, int nvec, long long N, int nx, int ny, int nz) {
  const long long total = (long long)nvec * N;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < total;
       j += (long long)gridDim.x * blockDim.x)
    out[j] = lz_face(j % N, nx, ny, nz) ? 0.0 : in[j];
}

// part[(q * nb + k) * gridDim.x + blockIdx.x]: this block's share of
// <Q_q, W_k>, q = blockIdx.y.
__global__ void __launch_bounds__(kT) k_lz_mdot(const double* __restrict__ Q, const double* __restrict__ W, int nb,
                                                 long long N, double* __restrict__ part) {
  const double* qv = Q + (long long)blockIdx.y * N;
  double acc[kMaxBlock] = {0.0, 0.0, 0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double x = qv[i];
#pragma unroll
    for (int k = 0; k < kMaxBlock; ++k)
      if (k < nb) acc[k] += x * W[k * N + i];
  }
  __shared__ double sh[kT / 32][kMaxBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kMaxBlock; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < nb) {
    double v = 0.0;
    for (int w = 0; w < kT / 32; ++w) v += sh[w][threadIdx.x];
    part[((long long)blockIdx.y * nb + threadIdx.x) * gridDim.x + blockIdx.x] = v;
  }
}

// out[j] = sum over the G block shares of entry j (fixed order); one warp per entry.
__global__ void k_lz_finish(const double* __restrict__ part, int G, double* __restrict__ out) {
  const int j = blockIdx.x;
  double v = 0.0;
  for (int x = threadIdx.x; x < G; x += 32) v += part[(long long)j * G + x];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) out[j] = v;
}

// W_k -= sum_q Q_q C[q * nb + k]
__global__ void __launch_bounds__(kT) k_lz_sub(double* __restrict__ W, int nb, const double* __restrict__ Q, int nq,
                                                const double* __restrict__ C, long long N) {
  extern __shared__ double sc[];
  for (int t = threadIdx.x; t < nq * nb; t += blockDim.x) sc[t] = C[t];
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double w[kMaxBlock];
#pragma unroll
    for (int k = 0; k < kMaxBlock; ++k) w[k] = k < nb ? W[k * N + i] : 0.0;
    for (int q = 0; q < nq; ++q) {
      const double x = Q[(long long)q * N + i];
#pragma unroll
      for (int k = 0; k < kMaxBlock; ++k)
        if (k < nb) w[k] -= x * sc[q * nb + k];
    }
#pragma unroll
    for (int k = 0; k < kMaxBlock; ++k)
      if (k < nb) W[k * N + i] = w[k];
  }
}

// out_c = sum_q Q_q S[q * ncol + c]   (out must not overlap Q)
__global__ void __launch_bounds__(kT) k_lz_combine(const double* __restrict__ Q, int nq, const double* __restrict__ S,
                                                    int ncol, double* __restrict__ out, long long N) {
  extern __shared__ double ss[];
  for (int t = threadIdx.x; t < nq * ncol; t += blockDim.x) ss[t] = S[t];
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double o[kMaxBlock] = {0.0, 0.0, 0.0, 0.0};
    for (int q = 0; q < nq; ++q) {
      const double x = Q[(long long)q * N + i];
#pragma unroll
      for (int c = 0; c < kMaxBlock; ++c)
        if (c < ncol) o[c] += x * ss[q * ncol + c];
    }
#pragma unroll
    for (int c = 0; c < kMaxBlock; ++c)
      if (c < ncol) out[c * N + i] = o[c];
  }
}

// Cholesky of the nb x nb Gram matrix G (row-major): G = R^T R with R upper
// triangular, and Rinv = R^-1.  A pivot below 1e-28 of the largest diagonal
// entry marks its direction dead (linearly dependent): R and Rinv get a zero
// there and flag is set.  One thread.
__global__ void k_lz_chol(const double* __restrict__ G, int nb, double* __restrict__ R, double* __restrict__ Rinv,
                          int* __restrict__ flag) {
  double r[kMaxBlock][kMaxBlock] = {}, ri[kMaxBlock][kMaxBlock] = {};
  double gmax = 0.0;
  for (int k = 0; k < nb; ++k) gmax = fmax(gmax, G[k * nb + k]);
  bool dead[kMaxBlock] = {};
  for (int j = 0; j < nb; ++j) {
    for (int i = 0; i <= j; ++i) {
      double s = G[i * nb + j];
      for (int l = 0; l < i; ++l) s -= r[l][i] * r[l][j];
      if (i == j) {
        if (s > 1e-28 * gmax && s > 0.0) {
          r[j][j] = sqrt(s);
        } else {
          r[j][j] = 0.0;
          dead[j] = true;
          *flag = 1;
        }
      } else {
        r[i][j] = dead[i] ? 0.0 : s / r[i][i];
      }
    }
  }
  // inverse of the upper triangle, column by column (dead rows/columns stay zero)
  for (int j = 0; j < nb; ++j) {
    if (dead[j]) continue;
    ri[j][j] = 1.0 / r[j][j];
    for (int i = j - 1; i >= 0; --i) {
      if (dead[i]) continue;
      double s = 0.0;
      for (int l = i + 1; l <= j; ++l) s += r[i][l] * ri[l][j];
      ri[i][j] = -s / r[i][i];
    }
  }
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      R[i * nb + j] = r[i][j];
      Rinv[i * nb + j] = ri[i][j];
    }
}

// C = A B (nb x nb, row-major); one thread.
__global__ void k_lz_matmul(const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C,
                            int nb) {
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      double s = 0.0;
      for (int l = 0; l < nb; ++l) s += A[i * nb + l] * B[l * nb + j];
      C[i * nb + j] = s;
    }
}

// Column block of the projected matrix: T[r * ldT + col0 + k] = C1 + C2.
__global__ void k_lz_store(double* __restrict__ T, int ldT, int col0, int nrows, const double* __restrict__ C1,
                           const double* __restrict__ C2, int nb) {
  for (int t = threadIdx.x; t < nrows * nb; t += blockDim.x) {
    const int r = t / nb, k = t % nb;
    T[(long long)r * ldT + col0 + k] = C1[t] + C2[t];
  }
}

// res = W_0 - lambda X_0 with lambda = *lam (device).
__global__ void k_lz_resid(const double* __restrict__ W, const double* __restrict__ X, const double* __restrict__ lam,
                           double* __restrict__ res, long long N) {
  const double l = *lam;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    res[i] = W[i] - l * X[i];
}

// Device allocations of one solve, freed on every exit path.
struct DevBufs {
  std::vector<void*> ptrs;
  template <typename T>
  T* get(size_t n) {
    void* p = nullptr;
    CDFT_CUDA(cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)));
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  ~DevBufs() {
    for (void* p : ptrs) cudaFree(p);
  }
};

struct PinnedBuf {
  double* p = nullptr;
  explicit PinnedBuf(size_t n) { CDFT_CUDA(cudaMallocHost(&p, sizeof(double) * std::max<size_t>(n, 1))); }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

}  // namespace

void symmetric_eigen(int n, const double* a_in, double* w, double* v) {
  std::vector<double> a(a_in, a_in + (size_t)n * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) v[i * n + j] = i == j ? 1.0 : 0.0;
  auto off = [&] {
    double s = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) s += a[i * n + j] * a[i * n + j];
    return s;
  };
  double scale = 0.0;
  for (int i = 0; i < n * n; ++i) scale = std::max(scale, std::abs(a[i]));
  for (int sweep = 0; sweep < 100 && off() > 1e-34 * scale * scale * n * n; ++sweep) {
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[p * n + q];
        if (std::abs(apq) < 1e-300) continue;
        // rotation annihilating a[p][q] (the classical Jacobi angle)
        const double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[k * n + p], vkq = v[k * n + q];
          v[k * n + p] = c * vkp - s * vkq;
          v[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  // sort ascending
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return a[x * n + x] < a[y * n + y]; });
  std::vector<double> vs((size_t)n * n);
  for (int c = 0; c < n; ++c) {
    w[c] = a[idx[c] * n + idx[c]];
    for (int r = 0; r < n; ++r) vs[r * n + c] = v[r * n + idx[c]];
  }
  std::copy(vs.begin(), vs.end(), v);
}

LanczosResult lanczos_lowest(Engine& hvp, const LanczosConfig& cfg, const double* rho, double* vec, bool use_guess,
                             cudaStream_t st) {
  const EvalParams& p = hvp.params();
  if (p.S != 1) throw Error(-1, "lanczos: single-species Hessians only");
  const int b = hvp.batch();
  if (b < 1 || b > kMaxBlock) throw Error(-1, "lanczos: block size 1..4 (the product engine's batch)");
  if (cfg.block != b) throw Error(-1, "lanczos: the block size must equal the product engine's batch");
  if (!rho || !vec) throw Error(-1, "lanczos: rho and vec are required");
  const int m = std::max(2, cfg.max_basis);
  const int check = std::max(1, cfg.check_interval);
  const long long N = p.N;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  int sms = 0, dev = 0;
  CDFT_CUDA(cudaGetDevice(&dev));
  CDFT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int G = (int)std::max<long long>(1, std::min<long long>((long long)sms * 4, (N + kT - 1) / kT));
  const int nmax = m * b;  // basis vectors before a restart
  const int ldT = nmax;

  DevBufs d;
  double* Q = d.get<double>((size_t)(m + 1) * b * N);
  double* W = d.get<double>((size_t)b * N);
  double* W1 = d.get<double>((size_t)b * N);
  double* X = d.get<double>((size_t)b * N);
  double* part = d.get<double>((size_t)nmax * b * G);
  double* C1 = d.get<double>((size_t)nmax * b);
  double* C2 = d.get<double>((size_t)nmax * b);
  double* T = d.get<double>((size_t)ldT * ldT);
  double* Rst = d.get<double>((size_t)m * b * b);
  double* Gm = d.get<double>((size_t)b * b);
  double* R1 = d.get<double>((size_t)b * b);
  double* Ri1 = d.get<double>((size_t)b * b);
  double* R2 = d.get<double>((size_t)b * b);
  double* Ri2 = d.get<double>((size_t)b * b);
  double* S = d.get<double>((size_t)nmax * b);
  double* sc = d.get<double>(8);
  int* flag = d.get<int>(1);
  CDFT_CUDA(cudaMemsetAsync(T, 0, sizeof(double) * ldT * ldT, st));
  CDFT_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
  PinnedBuf hT((size_t)ldT * ldT), hR((size_t)b * b + 8);

  // C[q * nb + k] = <A_q, B_k> for q < na, k < nb
  auto mdot = [&](const double* A, int na, const double* Bv, int nb, double* C) {
    k_lz_mdot<<<dim3(G, na), kT, 0, st>>>(A, Bv, nb, N, part);
    k_lz_finish<<<na * nb, 32, 0, st>>>(part, G, C);
  };
  // Q_out R = In (two Cholesky QR passes); R into Rout (may be null)
  auto orth = [&](const double* In, double* Qout, double* Rout) {
    mdot(In, b, In, b, Gm);
    k_lz_chol<<<1, 1, 0, st>>>(Gm, b, R1, Ri1, flag);
    k_lz_combine<<<G, kT, sizeof(double) * b * b, st>>>(In, b, Ri1, b, W1, N);
    mdot(W1, b, W1, b, Gm);
    k_lz_chol<<<1, 1, 0, st>>>(Gm, b, R2, Ri2, flag);
    k_lz_combine<<<G, kT, sizeof(double) * b * b, st>>>(W1, b, Ri2, b, Qout, N);
    if (Rout) k_lz_matmul<<<1, 1, 0, st>>>(R2, R1, Rout, b);
  };
  auto product = [&](const double* In, double* Out) {
    hvp.hvp_apply(In, Out, st);
    k_lz_faces<<<G, kT, 0, st>>>(Out, Out, b, N, nx, ny, nz);
  };

  // start block: the guess (faces zeroed) and / or seeded normal draws
  for (int k = 0; k < b; ++k) {
    if (k == 0 && use_guess)
      k_lz_faces<<<G, kT, 0, st>>>(vec, X, 1, N, nx, ny, nz);
    else
      k_lz_randn<<<G, kT, 0, st>>>(X + (size_t)k * N, N, cfg.seed + 7919ull * k, nx, ny, nz);
  }
  CDFT_CUDA(cudaGetLastError());
  orth(X, Q, nullptr);
  hvp.hvp_set_point(rho, st);

  LanczosResult res;
  std::vector<double> a, w, v;
  int j = 0;
  while (true) {
    double* Qj = Q + (size_t)j * b * N;
    product(Qj, W);
    ++res.iterations;
    const int nq = (j + 1) * b;
    // two passes of block classical Gram-Schmidt against the whole basis
    mdot(Q, nq, W, b, C1);
    k_lz_sub<<<G, kT, sizeof(double) * nq * b, st>>>(W, b, Q, nq, C1, N);
    mdot(Q, nq, W, b, C2);
    k_lz_sub<<<G, kT, sizeof(double) * nq * b, st>>>(W, b, Q, nq, C2, N);
    k_lz_store<<<1, 256, 0, st>>>(T, ldT, j * b, nq, C1, C2, b);
    orth(W, Q + (size_t)(j + 1) * b * N, Rst + (size_t)j * b * b);
    CDFT_CUDA(cudaGetLastError());
    const bool full = (j + 1 == m);
    const bool last = res.iterations >= cfg.max_iterations;
    if ((j + 1) % check != 0 && !full && !last) {
      ++j;
      continue;
    }
    // host check: the projected matrix and the last coupling
    CDFT_CUDA(cudaMemcpy2DAsync(hT.p, sizeof(double) * nq, T, sizeof(double) * ldT, sizeof(double) * nq, nq,
                                cudaMemcpyDeviceToHost, st));
    CDFT_CUDA(cudaMemcpyAsync(hR.p, Rst + (size_t)j * b * b, sizeof(double) * b * b, cudaMemcpyDeviceToHost, st));
    CDFT_CUDA(cudaStreamSynchronize(st));
    a.assign((size_t)nq * nq, 0.0);
    for (int r = 0; r < nq; ++r)
      for (int c = r; c < nq; ++c) a[(size_t)r * nq + c] = a[(size_t)c * nq + r] = hT.p[(size_t)r * nq + c];
    // a dead direction (a zero basis vector after a rank-deficient QR) has an
    // all-zero row: keep its spurious zero eigenvalue out of the lowest pairs
    for (int r = 0; r < nq; ++r) {
      bool zero = true;
      for (int c = 0; c < nq && zero; ++c) zero = a[(size_t)r * nq + c] == 0.0;
      if (zero) a[(size_t)r * nq + r] = 1e300;
    }
    w.assign(nq, 0.0);
    v.assign((size_t)nq * nq, 0.0);
    symmetric_eigen(nq, a.data(), w.data(), v.data());
    double rn = 0.0;
    for (int r = 0; r < b; ++r) {
      double t = 0.0;
      for (int c = 0; c < b; ++c) t += hR.p[r * b + c] * v[(size_t)(j * b + c) * nq + 0];
      rn += t * t;
    }
    rn = std::sqrt(rn);
    res.eigenvalue = w[0];
    res.residual = rn;
    const bool conv = rn < cfg.tolerance;
    if (conv || full || last) {
      // the b lowest Ritz vectors
      std::vector<double> s((size_t)nq * b);
      for (int r = 0; r < nq; ++r)
        for (int c = 0; c < b; ++c) s[(size_t)r * b + c] = v[(size_t)r * nq + c];
      CDFT_CUDA(cudaMemcpyAsync(S, s.data(), sizeof(double) * s.size(), cudaMemcpyHostToDevice, st));
      k_lz_combine<<<G, kT, sizeof(double) * nq * b, st>>>(Q, nq, S, b, X, N);
      CDFT_CUDA(cudaStreamSynchronize(st));  // s leaves scope
      if (conv || last) {
        res.converged = conv;
        break;
      }
      // restart from the lowest Ritz vectors
      orth(X, Q, nullptr);
      ++res.restarts;
      j = 0;
      continue;
    }
    ++j;
  }
  // the returned vector's own Rayleigh quotient and residual (one more product)
  product(X, W);
  mdot(X, 1, W, 1, sc);  // lambda = x . A x  (x is a unit vector)
  k_lz_resid<<<G, kT, 0, st>>>(W, X, sc, W1, N);
  mdot(W1, 1, W1, 1, sc + 1);
  mdot(X, 1, X, 1, sc + 2);
  CDFT_CUDA(cudaMemcpyAsync(hR.p, sc, sizeof(double) * 3, cudaMemcpyDeviceToHost, st));
  CDFT_CUDA(cudaMemcpyAsync(vec, X, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
  CDFT_CUDA(cudaStreamSynchronize(st));
  const double xx = hR.p[2];
  res.eigenvalue = hR.p[0] / xx;
  res.residual = std::sqrt(std::max(hR.p[1], 0.0) / xx);
  return res;
}

}  // namespace cdft
