// Device-resident drivers: FIRE2 minimisation, DDFT integrating-factor steps,
// Hessian-vector products.  See drivers.cuh.
#include "drivers.cuh"
#include "lanczos.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace cdft {

namespace {

constexpr int kBlock = 256;
constexpr int kRedTerms = 4;
constexpr int kOut = 8;  // reduced values per problem: two groups of kRedTerms

// Batched drivers: vector kernels take the problem from blockIdx.y, the
// single-thread control kernels from blockIdx.x (one block per problem).

__device__ __forceinline__ bool on_face(long long idx, int nx, int ny, int nz) {
  const int iz = (int)(idx % nz);
  const long long t = idx / nz;
  const int iy = (int)(t % ny);
  const int ix = (int)(t / ny);
  return ix == 0 || ix == nx - 1 || iy == 0 || iy == ny - 1 || iz == 0 || iz == nz - 1;
}

// block sums of up to kRedTerms values -> partials[problem][block][kRedTerms]
__device__ __forceinline__ void block_sum_store(double (&a)[kRedTerms], double* __restrict__ partials) {
  __shared__ double sh[32][kRedTerms];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < kRedTerms; ++t) {
    double v = a[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp][t] = v;
  }
  __syncthreads();
  if (threadIdx.x < kRedTerms) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sh[w][threadIdx.x];
    partials[((long long)blockIdx.y * gridDim.x + blockIdx.x) * kRedTerms + threadIdx.x] = v;
  }
}

// out[t] = sum_b partials[b][t], one warp per term; block i reduces problem i
// into out + i * kOut.
__global__ void k_finish_sums(const double* __restrict__ partials, int nblocks, double* __restrict__ out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  partials += (long long)blockIdx.x * nblocks * kRedTerms;
  out += blockIdx.x * kOut;
  if (warp >= kRedTerms) return;
  double v = 0.0;
  for (int b = lane; b < nblocks; b += 32) v += partials[b * kRedTerms + warp];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) out[warp] = v;
}

struct Vec {
  double* x;
  double* v;
  double* f;
  double* rho;
  double* grad;
  const double* dir;
  const double* vext;  // external field of the evaluations (B*N) or null
  long long N;
  int nx, ny, nz;
  double dv;
  int param;
  double rho_min, range;
};

// The vectors of problem blockIdx.y.
__device__ __forceinline__ Vec slice(Vec a) {
  const long long o = (long long)blockIdx.y * a.N;
  a.x += o;
  a.v += o;
  a.f += o;
  a.rho += o;
  a.grad += o;
  if (a.dir) a.dir += o;
  return a;
}

__device__ __forceinline__ double to_density(const Vec& a, double x) {
  if (a.param == kUnbounded) return a.rho_min + x * x;
  const double x2 = x * x;
  return a.rho_min + a.range * x2 / (1.0 + x2);
}

__device__ __forceinline__ double drho_dx(const Vec& a, double x) {
  if (a.param == kUnbounded) return 2.0 * x;
  const double x2 = x * x;
  const double den = (1.0 + x2) * (1.0 + x2);
  return 2.0 * a.range * x / den;
}

// minimization.hpp:63-78
__global__ void k_from_density(Vec a, const double* __restrict__ rho) {
  a = slice(a);
  rho += (long long)blockIdx.y * a.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
    double d = rho[i] - a.rho_min;
    double x;
    if (a.param == kUnbounded) {
      x = sqrt(d < 0.0 ? 0.0 : d);
    } else {
      const double hi = a.range * (1.0 - 1e-14);
      d = d < 0.0 ? 0.0 : (d > hi ? hi : d);
      x = sqrt(d / (a.range - d));
    }
    a.x[i] = x;
    a.v[i] = 0.0;
    a.rho[i] = to_density(a, x);
  }
}

// sums: [sum rho, sum_interior rho]
__global__ void k_density_sums(Vec a, double* __restrict__ partials) {
  a = slice(a);
  double s[kRedTerms] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
    const double r = a.rho[i];
    s[0] += r;
    if (!on_face(i, a.nx, a.ny, a.nz)) s[1] += r;
  }
  block_sum_store(s, partials);
}

__global__ void k_power(Vec a, double* __restrict__ partials) {
  a = slice(a);
  double s[kRedTerms] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x)
    s[0] += a.v[i] * a.f[i];
  block_sum_store(s, partials);
}

// fire.hpp:95-121: the power test, dt/alpha adaptation and uphill count.
__global__ void k_fire_control1(FireDevState* st, const double* __restrict__ sums, FireParams fp) {
  st += blockIdx.x;
  sums += blockIdx.x * kOut;
  if (threadIdx.x != 0 || !st->active) return;
  const double power = sums[0];
  st->dt_prev = st->dt;
  st->backtrack = 0;
  if (power > 0.0 || st->iteration == 0) {
    st->n_positive++;
    st->n_negative = 0;
    if (st->n_positive > fp.n_delay) {
      st->dt = fmin(st->dt * fp.f_inc, fp.dt_max);
      st->alpha *= fp.f_alpha;
    }
  } else {
    st->n_positive = 0;
    st->n_negative++;
    if (st->n_negative > fp.max_uphill) {
      st->uphill_error = 1;
      st->active = 0;
      return;
    }
    st->backtrack = 1;
    if (st->iteration > fp.n_delay) {
      st->dt = fmax(st->dt * fp.f_dec, fp.dt_min);
      st->alpha = fp.alpha_start;
    }
  }
}

// fire.hpp:110-126: backtrack (undo half a step with the old dt, kill v), then
// v += dt f; sums |v|^2.
__global__ void k_fire_vstep(Vec a, const FireDevState* __restrict__ st, double* __restrict__ partials) {
  a = slice(a);
  st += blockIdx.y;
  double s[kRedTerms] = {0, 0, 0, 0};
  if (st->active) {
    const double dt = st->dt, dtp = st->dt_prev;
    const bool bt = st->backtrack;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N;
         i += (long long)gridDim.x * blockDim.x) {
      double v = a.v[i];
      if (bt) {
        a.x[i] -= 0.5 * dtp * v;
        v = 0.0;
      }
      v += dt * a.f[i];
      a.v[i] = v;
      s[0] += v * v;
    }
  }
  block_sum_store(s, partials);
}

__global__ void k_fire_ratio(FireDevState* st, const double* __restrict__ sums) {
  st += blockIdx.x;
  sums += blockIdx.x * kOut;
  if (threadIdx.x != 0 || !st->active) return;
  const double v_norm = sqrt(sums[0]);
  const double f_norm = sqrt(st->f2);
  st->ratio = (f_norm > 0.0) ? v_norm / f_norm : -1.0;
}

// fire.hpp:137-148 then the parametrisation: mixing, x += dt v, rho = rho(x).
__global__ void k_fire_xstep(Vec a, const FireDevState* __restrict__ st) {
  a = slice(a);
  st += blockIdx.y;
  if (!st->active) return;
  const double dt = st->dt, al = st->alpha, ratio = st->ratio;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
    double v = a.v[i];
    if (ratio >= 0.0) v = (1.0 - al) * v + al * ratio * a.f[i];
    a.v[i] = v;
    const double x = a.x[i] + dt * v;
    a.x[i] = x;
    a.rho[i] = to_density(a, x);
  }
}

struct ComputeCfg {
  int mode;
  int homogeneous;
  double boundary_mass;
  double n_face;
};

// Fixed-mass rescale factor (minimization.hpp:193-197, saddle_point.hpp:448-463).
__global__ void k_scale_factor(FireDevState* st, const double* __restrict__ sums, ComputeCfg cc, double dv,
                               int force_compute) {
  st += blockIdx.x;
  sums += blockIdx.x * kOut;
  if (threadIdx.x != 0) return;
  if (!st->active && !force_compute) return;
  double scale = 1.0;
  if (cc.mode == kFixedMass) {
    const double mass = sums[0] * dv;
    if (mass > 0.0) scale = st->target_mass / mass;
  } else if (cc.mode == kSaddle) {
    const double m_int = sums[1] * dv;
    const double m_t = st->target_mass - cc.boundary_mass;
    if (m_int > 0.0 && m_t > 0.0) scale = m_t / m_int;
  }
  st->scale = scale;
}

__global__ void k_rescale(Vec a, const FireDevState* __restrict__ st, ComputeCfg cc, int force_compute) {
  a = slice(a);
  st += blockIdx.y;
  if ((!st->active && !force_compute) || cc.mode == kGrandPotential) return;
  const double sc = st->scale;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
    if (cc.mode == kFixedMass || !on_face(i, a.nx, a.ny, a.nz)) a.rho[i] *= sc;
  }
}

// sums [sum_face grad, sum_interior grad*rho, sum_face rho, sum_face grad*rho]
__global__ void k_post_sums(Vec a, double* __restrict__ partials) {
  a = slice(a);
  double s[kRedTerms] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
    const double g = a.grad[i], r = a.rho[i];
    if (on_face(i, a.nx, a.ny, a.nz)) {
      s[0] += g;
      s[2] += r;
      s[3] += g * r;
    } else {
      s[1] += g * r;
    }
  }
  block_sum_store(s, partials);
}

// The Lagrange multiplier (minimization.hpp:212-217, saddle_point.hpp:472-480).
__global__ void k_post_control(FireDevState* st, const double* __restrict__ sums, ComputeCfg cc) {
  st += blockIdx.x;
  sums += blockIdx.x * kOut;
  if (threadIdx.x != 0) return;
  const double bavg = (cc.n_face > 0.0) ? sums[0] / cc.n_face : 0.0;
  st->bavg = bavg;
  double lam = 0.0;
  if (cc.mode == kFixedMass) {
    // <grad_b, rho> with grad_b the boundary-treated gradient
    const double face = cc.homogeneous ? bavg * sums[2] : sums[3];
    lam = (sums[1] + face) / st->target_mass;
  } else if (cc.mode == kSaddle) {
    const double m_t = st->target_mass - cc.boundary_mass;
    lam = sums[1];
    if (m_t > 0.0) lam /= m_t;
  }
  st->lambda = lam;
}

// Boundary treatment, Lagrange term and chain rule: f = -grad * drho/dx
// (saddle: the projection follows).  sums [|f|^2, dir . f_alias].
__global__ void k_post_apply(Vec a, const FireDevState* __restrict__ st, ComputeCfg cc,
                             double* __restrict__ partials) {
  a = slice(a);
  st += blockIdx.y;
  double s[kRedTerms] = {0, 0, 0, 0};
  const double bavg = st->bavg;
  const double lam = st->lambda;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
    double g = a.grad[i];
    const bool face = on_face(i, a.nx, a.ny, a.nz);
    if (cc.mode == kSaddle) {
      g = face ? 0.0 : g - lam * a.dv;
    } else {
      if (cc.homogeneous && face) g = bavg;
      if (cc.mode == kFixedMass) g -= lam * a.dv;
    }
    const double fa = g * drho_dx(a, a.x[i]);  // transform_force (minimization.hpp:82-99)
    if (cc.mode == kSaddle) {
      a.f[i] = fa;  // projected by k_project
      s[1] += a.dir[i] * fa;
    } else {
      a.f[i] = -fa;
      s[0] += fa * fa;
    }
  }
  block_sum_store(s, partials);
}

// saddle_point.hpp:490-492: f_alias -= (dir . f_alias) dir; f = -f_alias.
__global__ void k_project(Vec a, const double* __restrict__ sums_in, double* __restrict__ partials) {
  a = slice(a);
  sums_in += blockIdx.y * kOut;
  double s[kRedTerms] = {0, 0, 0, 0};
  const double proj = sums_in[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
    const double fa = a.f[i] - proj * a.dir[i];
    a.f[i] = -fa;
    s[0] += fa * fa;
  }
  block_sum_store(s, partials);
}

// fire.hpp:150-162 and minimization.hpp:431-434: energy, rms force, the
// convergence monitor and the iteration counter.
__global__ void k_fire_finalize(FireDevState* st, const double* __restrict__ sums, const double* __restrict__ scal,
                                FireParams fp, double n_dof, double volume, int use_monitor, int initial) {
  st += blockIdx.x;
  sums += blockIdx.x * kOut;
  scal += blockIdx.x * kScalarCount;
  if (threadIdx.x != 0) return;
  if (!initial && !st->active) return;
  const double f2 = sums[0];
  st->f2 = f2;
  const double old_e = st->energy;
  st->energy = scal[1];
  st->free_energy = scal[0];
  st->rms_force = sqrt(f2 / n_dof);
  if (initial) {
    st->converged = use_monitor ? 0 : (st->rms_force < fp.force_tolerance);
    st->active = (!st->converged && fp.max_steps > 0) ? 1 : 0;
    return;
  }
  st->iteration++;
  if (use_monitor) {
    st->vv = st->vv * 0.9 + 0.1 * (fabs(st->energy - old_e) / st->dt);
    st->monitor = fabs(st->vv / volume);
    st->converged = st->monitor < fp.force_tolerance;
  } else {
    st->converged = st->rms_force < fp.force_tolerance;
  }
  if (st->converged || st->iteration >= fp.max_steps) st->active = 0;
}

// The FP64 engine takes over a minimisation whose problems converged under
// the mixed-precision forces: they continue until the FP64 forces meet the
// tolerance too (problems stopped by an uphill error or the step limit stay
// stopped).
__global__ void k_fire_reactivate(FireDevState* st, int max_steps) {
  st += blockIdx.x;
  if (threadIdx.x != 0) return;
  if (!st->active && st->converged && !st->uphill_error && st->iteration < max_steps) {
    st->converged = 0;
    st->active = 1;
  }
}

// ---------------------------------------------------------------- DDFT

// dynamics.hpp:135-206: R = div(rho grad(force/dV)) - lap(rho).
__global__ void k_ddft_rhs(const double* __restrict__ rho, const double* __restrict__ force, double* __restrict__ out,
                           int nx, int ny, int nz, double dx, double inv_dv) {
  const long long N = (long long)nx * ny * nz;
  const double D = 0.5 / (dx * dx);
  const double L = 1.0 / (dx * dx);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(p % nz);
    const long long t = p / nz;
    const int iy = (int)(t % ny);
    const int ix = (int)(t / ny);
    const long long nyz = (long long)ny * nz;
    const long long ixp = ((ix + 1) % nx) * nyz, ixm = ((ix - 1 + nx) % nx) * nyz, ix0 = ix * nyz;
    const long long iyp = ((iy + 1) % ny) * (long long)nz, iym = ((iy - 1 + ny) % ny) * (long long)nz,
                    iy0 = iy * (long long)nz;
    const int izp = (iz + 1) % nz, izm = (iz - 1 + nz) % nz;
    const double d0 = rho[p];
    const double x0 = force[p] * inv_dv;
    const long long px = ixp + iy0 + iz, mx = ixm + iy0 + iz, py = ix0 + iyp + iz, my = ix0 + iym + iz,
                    pz = ix0 + iy0 + izp, mz = ix0 + iy0 + izm;
    const double g = D * ((rho[px] + d0) * (force[px] * inv_dv - x0) - (d0 + rho[mx]) * (x0 - force[mx] * inv_dv)) +
                     D * ((rho[py] + d0) * (force[py] * inv_dv - x0) - (d0 + rho[my]) * (x0 - force[my] * inv_dv)) +
                     D * ((rho[pz] + d0) * (force[pz] * inv_dv - x0) - (d0 + rho[mz]) * (x0 - force[mz] * inv_dv));
    const double lap = L * (rho[px] + rho[mx] - 2.0 * d0) + L * (rho[py] + rho[my] - 2.0 * d0) +
                       L * (rho[pz] + rho[mz] - 2.0 * d0);
    out[p] = g - lap;
  }
}

// Device-side control state of one integrating-factor step.
struct DdftDevState {
  double dt;               // the time step of the current attempt
  double deviation;        // max |d1_new - d1| of the last iteration
  double min_density;      // min d1_new of the last iteration
  double refine_deviation; // deviation of the last FP64 refinement iteration
  int it;                  // iterations of the current attempt
  int total_it;            // iterations of the step
  int restarts;
  int status;              // 0 iterating, 1 converged, 2 gave up
  int copy_back;           // the attempt restarts: d1 <- rho
  int pad;
};

// dynamics.hpp:247-287: work = U0 rho0_k + U1 R0_k + U2 (R1_k - R0_k), at
// the control state's dt.
__global__ void k_ddft_propagate(const double2* __restrict__ rho0k, const double2* __restrict__ r0k,
                                 double2* __restrict__ r1k_work, const double* __restrict__ lam, int nx, int ny,
                                 int nzh, const DdftDevState* __restrict__ st) {
  const double dt = st->dt;
  const long long Nk = (long long)nx * ny * nzh;
  for (long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x; pos < Nk;
       pos += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(pos % nzh);
    const long long t = pos / nzh;
    const int iy = (int)(t % ny);
    const int ix = (int)(t / ny);
    const double Lambda = lam[ix] + lam[nx + iy] + lam[nx + ny + iz];
    const double ex = exp(lam[ix] * dt) * exp(lam[nx + iy] * dt) * exp(lam[nx + ny + iz] * dt);
    const double U0 = ex;
    const double U1 = (pos == 0) ? dt : (ex - 1.0) / Lambda;
    const double U2 = (pos == 0) ? dt / 2.0 : (ex - 1.0 - dt * Lambda) / (Lambda * Lambda * dt);
    const double2 a = rho0k[pos], b = r0k[pos], c = r1k_work[pos];
    r1k_work[pos] = make_double2(U0 * a.x + U1 * b.x + U2 * (c.x - b.x), U0 * a.y + U1 * b.y + U2 * (c.y - b.y));
  }
}

// d1_new = work / N; sums [max |d1 - d1_new|, min d1_new] via partial max/min.
__global__ void k_ddft_update(const double* __restrict__ work, double* __restrict__ d1, long long N, double inv_n,
                              double* __restrict__ partials) {
  double mx = 0.0, mn = 1e300;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double nv = work[i] * inv_n;
    const double dev = fabs(d1[i] - nv);
    mx = dev > mx ? dev : mx;
    mn = nv < mn ? nv : mn;
    d1[i] = nv;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  __shared__ double smx[32], smn[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smx[warp] = mx;
    smn[warp] = mn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      mx = fmax(mx, smx[w]);
      mn = fmin(mn, smn[w]);
    }
    partials[blockIdx.x * 2 + 0] = fmax(mx, smx[0]);
    partials[blockIdx.x * 2 + 1] = fmin(mn, smn[0]);
  }
}

__global__ void k_maxmin_finish(const double* __restrict__ partials, int nb, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double mx = 0.0, mn = 1e300;
  for (int b = 0; b < nb; ++b) {
    mx = fmax(mx, partials[2 * b]);
    mn = fmin(mn, partials[2 * b + 1]);
  }
  out[0] = mx;
  out[1] = mn;
}

// Start of a step's fixed-point loop (dt is set by the host beforehand).
__global__ void k_ddft_begin(DdftDevState* st) {
  if (threadIdx.x != 0) return;
  st->deviation = 1e30;
  st->min_density = 0.0;
  st->refine_deviation = 0.0;
  st->it = st->total_it = st->restarts = st->status = st->copy_back = 0;
}

// One fixed-point iteration's decision (dynamics.hpp:362-389): a negative
// density or a growing deviation restarts the attempt at dt / 10 from rho, as
// does a deviation still above the tolerance after fp_max iterations; a
// deviation below it ends the loop.  With use_cond the loop's conditional
// node continues while the status is 0.  After max_restarts restarts the
// step gives up (status 2) with the last iterate.
__global__ void k_ddft_control(DdftDevState* st, const double* __restrict__ red, double tol, int fp_max,
                               int max_restarts, cudaGraphConditionalHandle cond, int use_cond) {
  if (threadIdx.x != 0) return;
  const double old = st->deviation;
  const double dev = red[0], mn = red[1];
  st->it += 1;
  st->total_it += 1;
  st->deviation = dev;
  st->min_density = mn;
  st->copy_back = 0;
  bool restart = false;
  if (mn < 0.0 || (st->it > 1 && dev > old))
    restart = true;
  else if (dev < tol)
    st->status = 1;
  else if (st->it >= fp_max)
    restart = true;
  if (restart) {
    st->restarts += 1;
    if (st->restarts >= max_restarts) {
      st->status = 2;
    } else {
      st->dt /= 10.0;
      st->it = 0;
      st->deviation = 1e30;
      st->copy_back = 1;
    }
  }
  if (use_cond) cudaGraphSetConditional(cond, st->status == 0 ? 1u : 0u);
}

// d1 <- rho when the attempt restarts.
__global__ void k_ddft_copy_back(const DdftDevState* __restrict__ st, const double* __restrict__ rho,
                                 double* __restrict__ d1, long long N) {
  if (!st->copy_back) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    d1[i] = rho[i];
}

__global__ void k_ddft_refine_record(DdftDevState* st, const double* __restrict__ red) {
  if (threadIdx.x == 0) st->refine_deviation = red[0];
}

// ------------------------------------------------------------------- HVP

// hv = (f_eps - f0) / eps with the fixed boundary applied to both.
__global__ void k_fd_hvp(const double* __restrict__ f_eps, const double* __restrict__ f0, double* __restrict__ hv,
                         long long N, double inv_eps, int nx, int ny, int nz, int boundary) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const bool zero = boundary && on_face(i, nx, ny, nz);
    hv[i] = zero ? 0.0 : (f_eps[i] - f0[i]) * inv_eps;
  }
}

__global__ void k_axpy_into(const double* __restrict__ x, double a, const double* __restrict__ y,
                            double* __restrict__ out, long long N) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    out[i] = y[i] + a * x[i];
}

__global__ void k_fixed_boundary(double* __restrict__ f, long long N, int nx, int ny, int nz) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    if (on_face(i, nx, ny, nz)) f[i] = 0.0;
}

__global__ void k_dot(const double* __restrict__ a, const double* __restrict__ b, long long n,
                      double* __restrict__ partials) {
  double s[kRedTerms] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s[0] += a[i] * b[i];
  block_sum_store(s, partials);
}

__global__ void k_axpby(double a, const double* __restrict__ x, double b, double* __restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

// Seeded standard normal draws (splitmix64 counter hash + Box-Muller).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void k_randn(double* __restrict__ out, long long n, unsigned long long seed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long a = mix64(seed * 0x100000001b3ull + 2 * i);
    const unsigned long long b = mix64(seed * 0x100000001b3ull + 2 * i + 1);
    const double u1 = ((a >> 11) + 1.0) * (1.0 / 9007199254740993.0);  // (0, 1]
    const double u2 = (b >> 11) * (1.0 / 9007199254740992.0);
    out[i] = sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
  }
}

// out = a*x + b*y + c*z (any of y, z may be null)
__global__ void k_lincomb(double* __restrict__ out, double a, const double* __restrict__ x, double b,
                          const double* __restrict__ y, double c, const double* __restrict__ z, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = a * x[i];
    if (y) v += b * y[i];
    if (z) v += c * z[i];
    out[i] = v;
  }
}

// dir = vec * drho/dx at x = x(rho) (saddle_point.hpp:424-426)
__global__ void k_dir_alias(const double* __restrict__ vec, const double* __restrict__ rho, double* __restrict__ out,
                            long long n, double rho_min) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = rho[i] - rho_min;
    const double x = sqrt(d < 0.0 ? 0.0 : d);
    out[i] = vec[i] * 2.0 * x;
  }
}

__global__ void k_face_sum(const double* __restrict__ rho, long long n, int nx, int ny, int nz,
                           double* __restrict__ partials) {
  double s[kRedTerms] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (on_face(i, nx, ny, nz)) s[0] += rho[i];
  block_sum_store(s, partials);
}

// --------------------------------------------------- split / CN DDFT steps

// |k|^2 of half-spectrum index pos (dynamics.hpp:310-318: the wavevector of
// grid.hpp with the Nyquist index positive).
__device__ __forceinline__ double k_squared(long long pos, int nx, int ny, int nzh, int nz, double dx) {
  const int iz = (int)(pos % nzh);
  const long long t = pos / nzh;
  const int iy = (int)(t % ny);
  const int ix = (int)(t / ny);
  const double kx = 2.0 * 3.14159265358979323846 / (nx * dx) * (double)(ix <= nx / 2 ? ix : ix - nx);
  const double ky = 2.0 * 3.14159265358979323846 / (ny * dx) * (double)(iy <= ny / 2 ? iy : iy - ny);
  const double kz = 2.0 * 3.14159265358979323846 / (nz * dx) * (double)iz;
  return kx * kx + ky * ky + kz * kz;
}

// work *= sqrt(exp(-D k^2 dt)) (the half propagator of dynamics.hpp:426).
__global__ void k_half_diffusion(double2* __restrict__ work, int nx, int ny, int nzh, int nz, double dx, double D,
                                 double dt) {
  const long long Nk = (long long)nx * ny * nzh;
  for (long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x; pos < Nk;
       pos += (long long)gridDim.x * blockDim.x) {
    const double h = sqrt(exp(-D * k_squared(pos, nx, ny, nzh, nz, dx) * dt));
    const double2 v = work[pos];
    work[pos] = make_double2(v.x * h, v.y * h);
  }
}

// out = max(in * scale + dt * add, min_density) (add may be null).
__global__ void k_scale_clamp(const double* __restrict__ in, const double* __restrict__ add, double* __restrict__ out,
                              long long N, double scale, double dt, double min_density) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double v = in[i] * scale;
    if (add) v += dt * add[i];
    out[i] = v < min_density ? min_density : v;
  }
}

// The Crank-Nicolson update of dynamics.hpp:518-521 in k-space:
// wk = ((1 - a) rho0_k + dt/2 (R0_k + R1_k)) / (1 + a), a = D k^2 dt / 2.
__global__ void k_cn_combine(const double2* __restrict__ rho0k, const double2* __restrict__ r0k,
                             double2* __restrict__ r1k_work, int nx, int ny, int nzh, int nz, double dx, double D,
                             double dt) {
  const long long Nk = (long long)nx * ny * nzh;
  for (long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x; pos < Nk;
       pos += (long long)gridDim.x * blockDim.x) {
    const double a = D * k_squared(pos, nx, ny, nzh, nz, dx) * dt * 0.5;
    const double cm = 1.0 - a, cpi = 1.0 / (1.0 + a);
    const double2 r0 = rho0k[pos], q0 = r0k[pos], q1 = r1k_work[pos];
    r1k_work[pos] = make_double2((cm * r0.x + (dt * 0.5) * (q0.x + q1.x)) * cpi,
                                 (cm * r0.y + (dt * 0.5) * (q0.y + q1.y)) * cpi);
  }
}

// d1_new = max(work / N, min); partial max |d1_new - d1|; d1 = d1_new.
__global__ void k_cn_update(const double* __restrict__ work, double* __restrict__ d1, long long N, double inv_n,
                            double min_density, double* __restrict__ partials) {
  double mx = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double nv = work[i] * inv_n;
    nv = nv < min_density ? min_density : nv;
    const double dev = fabs(nv - d1[i]);
    mx = dev > mx ? dev : mx;
    d1[i] = nv;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  __shared__ double smx[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smx[warp] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, smx[w]);
    partials[blockIdx.x * 2 + 0] = fmax(mx, smx[0]);
    partials[blockIdx.x * 2 + 1] = 0.0;
  }
}

__global__ void k_reservoir_fill(double* __restrict__ rho, const unsigned char* __restrict__ mask, long long N,
                                 double value) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    if (mask[i]) rho[i] = value;
}

// ------------------------------------------------------------------ Picard

struct PicardDevState {
  double omega, omega_prev, residual, target_mass, scale;
  int iter, active, converged, apply;
};

// sums [sum f^2] of problem blockIdx.y
__global__ void k_sum_sq(const double* __restrict__ f, long long N, double* __restrict__ partials) {
  f += (long long)blockIdx.y * N;
  double s[kRedTerms] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    s[0] += f[i] * f[i];
  block_sum_store(s, partials);
}

// picard.hpp:81-106: residual, the two convergence tests, Omega bookkeeping.
__global__ void k_picard_control(PicardDevState* st, const double* __restrict__ sums, const double* __restrict__ scal,
                                 double n_dof, double tol) {
  st += blockIdx.x;
  sums += blockIdx.x * kOut;
  scal += blockIdx.x * kScalarCount;
  if (threadIdx.x != 0 || !st->active) return;
  st->omega = scal[1];
  st->residual = sqrt(sums[0] / n_dof);
  const bool force_conv = st->residual < tol;
  const bool omega_conv = st->iter > 0 && fabs(st->omega - st->omega_prev) < tol;
  if (force_conv || omega_conv) {
    st->converged = 1;
    st->active = 0;
    return;
  }
  st->omega_prev = st->omega;
}

// picard.hpp:108-111: rho *= exp(-mixing f / dV), clamped at min_density.
__global__ void k_picard_update(double* __restrict__ rho, const double* __restrict__ f,
                                const PicardDevState* __restrict__ st, long long N, double mixing_over_dv,
                                double min_density) {
  st += blockIdx.y;
  if (!st->active) return;
  rho += (long long)blockIdx.y * N;
  f += (long long)blockIdx.y * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double v = rho[i] * exp(-mixing_over_dv * f[i]);
    rho[i] = v < min_density ? min_density : v;
  }
}

// sums [sum (rho - background)] of problem blockIdx.y (background may be null)
__global__ void k_excess_sum(const double* __restrict__ rho, const double* __restrict__ bg, long long N,
                             double* __restrict__ partials) {
  rho += (long long)blockIdx.y * N;
  if (bg) bg += (long long)blockIdx.y * N;
  double s[kRedTerms] = {0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    s[0] += rho[i] - (bg ? bg[i] : 0.0);
  block_sum_store(s, partials);
}

// minimization.hpp:169-175: the mass rescale of the excess over the background.
__global__ void k_picard_mass(PicardDevState* st, const double* __restrict__ sums, double dv) {
  st += blockIdx.x;
  sums += blockIdx.x * kOut;
  if (threadIdx.x != 0) return;
  const double mass = sums[0] * dv;
  st->apply = (st->active && fabs(mass) > 1e-30) ? 1 : 0;
  st->scale = st->apply ? st->target_mass / mass : 1.0;
}

__global__ void k_picard_rescale(double* __restrict__ rho, const double* __restrict__ bg,
                                 const PicardDevState* __restrict__ st, long long N, double min_density) {
  st += blockIdx.y;
  if (!st->apply) return;
  rho += (long long)blockIdx.y * N;
  if (bg) bg += (long long)blockIdx.y * N;
  const double sc = st->scale;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double b = bg ? bg[i] : 0.0;
    const double v = b + sc * (rho[i] - b);
    rho[i] = v < min_density ? min_density : v;
  }
}

__global__ void k_picard_count(PicardDevState* st) {
  st += blockIdx.x;
  if (threadIdx.x == 0 && st->active) st->iter++;
}

// Symmetric eigen-decomposition of a small matrix (cyclic Jacobi); returns
// the eigenvector of the smallest eigenvalue (the reference takes column 0
// of arma::eig_sym, saddle_point.hpp:251-254).
void smallest_eigvec(int n, double A[3][3], double* vec, double* val) {
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) off += A[i][j] * A[i][j];
    if (off < 1e-300) break;
    for (int pq = 0; pq < n; ++pq)
      for (int q = pq + 1; q < n; ++q) {
        const int pp = pq;
        if (std::abs(A[pp][q]) < 1e-300) continue;
        const double theta = (A[q][q] - A[pp][pp]) / (2.0 * A[pp][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = A[k][pp], akq = A[k][q];
          A[k][pp] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A[pp][k], aqk = A[q][k];
          A[pp][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[k][pp], vkq = V[k][q];
          V[k][pp] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int m = 0;
  for (int i = 1; i < n; ++i)
    if (A[i][i] < A[m][m]) m = i;
  for (int k = 0; k < n; ++k) vec[k] = V[k][m];
  *val = A[m][m];
}

}  // namespace

Drivers::Drivers(Engine& engine) : eng_(engine) {
  if (engine.species() != 1) throw Error(-1, "drivers: the minimiser, DDFT and saddle drivers are single-species");
  N_ = engine.points();
  B_ = engine.batch();
  const size_t BN = (size_t)B_ * N_;
  auto al = [&](double** p, size_t n) { CDFT_CUDA(cudaMalloc(p, sizeof(double) * n)); };
  al(&x_, BN);
  al(&v_, BN);
  al(&f_, BN);
  al(&grad_, BN);
  al(&tmp_, N_);
  al(&tmp2_, N_);
  al(&scalars_, (size_t)B_ * kScalarCount);
  int sms = 0, dev = 0;
  CDFT_CUDA(cudaGetDevice(&dev));
  CDFT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // about 8 CTAs per SM in total, shared by the B problems
  const long long all = std::max<long long>(1, std::min<long long>((long long)sms * 8, ((long long)BN + kBlock - 1) / kBlock));
  grid_ = (int)std::max<long long>(1, (all + B_ - 1) / B_);
  al(&red_, (size_t)B_ * grid_ * kRedTerms + 64);
  al(&red_out_, std::max<size_t>(64, (size_t)B_ * kOut));
  CDFT_CUDA(cudaMalloc(&st_, sizeof(FireDevState) * B_));
  CDFT_CUDA(cudaMallocHost(&st_host_, sizeof(FireDevState) * B_));
  CDFT_CUDA(cudaMallocHost(&host_pin_, sizeof(double) * 64));
}

Drivers::~Drivers() {
  for (void* p : {(void*)x_, (void*)v_, (void*)f_, (void*)grad_, (void*)tmp_, (void*)tmp2_, (void*)scalars_,
                  (void*)red_, (void*)red_out_, (void*)st_, ddft_k_, (void*)lam_, fft_work_, tan_})
    if (p) cudaFree(p);
  for (double* p : ev_)
    if (p) cudaFree(p);
  if (st_host_) cudaFreeHost(st_host_);
  for (int i = 0; i < 2; ++i) {
    if (snap_stage_[i]) cudaFree(snap_stage_[i]);
    if (snap_ready_[i]) cudaEventDestroy(snap_ready_[i]);
    if (snap_done_[i]) cudaEventDestroy(snap_done_[i]);
  }
  if (copy_stream_) cudaStreamDestroy(copy_stream_);
  reset_step_graph();
  reset_fp_graph();
  if (graph_stream_) cudaStreamDestroy(graph_stream_);
  for (cudaEvent_t e : graph_ev_)
    if (e) cudaEventDestroy(e);
  if (host_pin_) cudaFreeHost(host_pin_);
  if (ddft_ready_) {
    cufftDestroy(plan_r2c_);
    cufftDestroy(plan_c2r_);
  }
}

double Drivers::dot(const double* a, const double* b, long long n, cudaStream_t stream) {
  k_dot<<<grid_, kBlock, 0, stream>>>(a, b, n, red_);
  k_finish_sums<<<1, 32 * kRedTerms, 0, stream>>>(red_, grid_, red_out_);
  CDFT_CUDA(cudaMemcpyAsync(host_pin_, red_out_, sizeof(double), cudaMemcpyDeviceToHost, stream));
  CDFT_CUDA(cudaStreamSynchronize(stream));
  return host_pin_[0];
}

void Drivers::axpby(double a, const double* x, double b, double* y, long long n, cudaStream_t stream) {
  k_axpby<<<grid_, kBlock, 0, stream>>>(a, x, b, y, n);
  CDFT_CUDA(cudaGetLastError());
}

double Drivers::force(const double* rho, double* f, double mu, int boundary, cudaStream_t stream) {
  eng_.evaluate(rho, nullptr, &mu, f, scalars_, stream);
  const EvalParams& p = eng_.params();
  if (boundary) k_fixed_boundary<<<grid_, kBlock, 0, stream>>>(f, N_, p.nx, p.ny, p.nz);
  CDFT_CUDA(cudaMemcpyAsync(host_pin_, scalars_, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
  CDFT_CUDA(cudaStreamSynchronize(stream));
  return host_pin_[1];
}

void Drivers::hvp_fd(const double* rho, const double* force_at_rho, const double* v, double* hv, double eps,
                     double mu, int boundary, cudaStream_t stream) {
  const EvalParams& p = eng_.params();
  k_axpy_into<<<grid_, kBlock, 0, stream>>>(v, eps, rho, tmp_, N_);  // rho + eps v
  eng_.evaluate(tmp_, nullptr, &mu, tmp2_, scalars_, stream);
  k_fd_hvp<<<grid_, kBlock, 0, stream>>>(tmp2_, force_at_rho, hv, N_, 1.0 / eps, p.nx, p.ny, p.nz, boundary);
  CDFT_CUDA(cudaGetLastError());
}

void Drivers::hvp_exact(const double* rho, const double* v, double* hv, double mu, int boundary,
                        cudaStream_t stream) {
  eng_.hvp(rho, v, &mu, hv, stream);
  const EvalParams& p = eng_.params();
  if (boundary) k_fixed_boundary<<<grid_, kBlock, 0, stream>>>(hv, N_, p.nx, p.ny, p.nz);
  CDFT_CUDA(cudaGetLastError());
}

FireResult Drivers::fire_minimize(const FireConfig& cfg, double* rho, const double* direction, cudaStream_t stream,
                                  Engine* refine, double refine_switch) {
  if (B_ != 1) throw Error(-1, "fire_minimize: needs an engine with batch 1");
  if (cfg.mode == kSaddle && !direction) throw Error(-1, "fire_minimize: saddle mode needs a direction");
  if (cfg.mode == kFixedMass && !(cfg.target_mass > 0.0)) throw Error(-1, "fire_minimize: target mass must be > 0");
  return fire_run(cfg, &cfg.mu, &cfg.target_mass, rho, direction, stream, refine, refine_switch)[0];
}

std::vector<FireResult> Drivers::fire_minimize_batch(const FireConfig& cfg, const double* mu, const double* mass,
                                                     double* rho, cudaStream_t stream, Engine* refine,
                                                     double refine_switch) {
  if (cfg.mode == kSaddle) throw Error(-1, "fire_minimize_batch: the saddle mode is single-problem");
  if (!mu) throw Error(-1, "fire_minimize_batch: mu is required");
  std::vector<double> m(B_, 0.0);
  if (cfg.mode == kFixedMass) {
    if (!mass) throw Error(-1, "fire_minimize_batch: fixed mass needs a target mass per problem");
    for (int b = 0; b < B_; ++b) {
      if (!(mass[b] > 0.0)) throw Error(-1, "fire_minimize_batch: target masses must be > 0");
      m[b] = mass[b];
    }
  }
  if (refine && refine->batch() != B_) throw Error(-1, "fire_minimize_batch: the refine engine needs the same batch");
  return fire_run(cfg, mu, m.data(), rho, nullptr, stream, refine, refine_switch);
}

// FIRE2 for the B problems of the engine: each step is a fixed sequence of
// launches over all problems; every control decision is taken per problem
// on the device (fire.hpp:86-165, minimization.hpp:182-354).
namespace {
std::atomic<bool> g_step_graphs{true};
}  // namespace

void set_step_graphs(bool on) { g_step_graphs.store(on); }
bool step_graphs() { return g_step_graphs.load(); }

void Drivers::ensure_graph_stream() {
  if (graph_stream_) return;
  CDFT_CUDA(cudaStreamCreateWithFlags(&graph_stream_, cudaStreamNonBlocking));
  for (cudaEvent_t& e : graph_ev_) CDFT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

void Drivers::reset_fp_graph() {
  if (fp_exec_) cudaGraphExecDestroy(fp_exec_);
  if (fp_graph_) cudaGraphDestroy(fp_graph_);
  fp_exec_ = nullptr;
  fp_graph_ = nullptr;
}

void Drivers::reset_step_graph() {
  if (step_exec_) cudaGraphExecDestroy(step_exec_);
  if (step_graph_) cudaGraphDestroy(step_graph_);
  step_exec_ = nullptr;
  step_graph_ = nullptr;
  step_key_ = nullptr;
}

// The minimiser loop on the caller's stream, or (step graphs on, stage timing
// off) on the driver's own stream joined to the caller's by events at entry
// and exit: stream capture needs a stream other than the legacy default one.
std::vector<FireResult> Drivers::fire_run(const FireConfig& cfg, const double* mu, const double* mass, double* rho,
                                          const double* direction, cudaStream_t stream, Engine* refine,
                                          double refine_switch) {
  const bool graphs = step_graphs() && !eng_.stage_timing_on() && !(refine && refine->stage_timing_on());
  if (!graphs) return fire_loop(cfg, mu, mass, rho, direction, stream, refine, refine_switch, false);
  ensure_graph_stream();
  CDFT_CUDA(cudaEventRecord(graph_ev_[0], stream));
  CDFT_CUDA(cudaStreamWaitEvent(graph_stream_, graph_ev_[0], 0));
  std::vector<FireResult> out;
  try {
    out = fire_loop(cfg, mu, mass, rho, direction, graph_stream_, refine, refine_switch, true);
  } catch (...) {
    reset_step_graph();
    cudaEventRecord(graph_ev_[1], graph_stream_);
    cudaStreamWaitEvent(stream, graph_ev_[1], 0);
    throw;
  }
  CDFT_CUDA(cudaEventRecord(graph_ev_[1], graph_stream_));
  CDFT_CUDA(cudaStreamWaitEvent(stream, graph_ev_[1], 0));
  return out;
}

// State of one FIRE run of this driver (all problems of its engine): the
// kernel arguments, the engine evaluating and the host's step count.
struct FireRun {
  FireConfig cfg;
  Vec a;
  ComputeCfg cc;
  double volume = 0.0;
  std::vector<double> mu_compute, mu_final;
  Engine* eng = nullptr;
  Engine* refine = nullptr;
  double refine_switch = 10.0;
  bool refining = false;
  int steps = 0;
  bool done = false;
  // stagnation of the mixed-precision run: the best convergence measure seen
  // at a check and the checks since it last improved by 10%
  double best_metric = 0.0;
  int stalled_checks = 0;
};

// Checks without a 10% improvement after which the FP64 engine takes over:
// mixed-precision forces have a noise floor, and a tolerance below it is
// reached only with FP64 forces.
constexpr int kStallChecks = 8;

// rescale (fixed mass / saddle), evaluate, post-process into f
void Drivers::fire_compute(int initial, cudaStream_t stream) {
  FireRun& r = *run_;
  const EvalParams& p = eng_.params();
  const int B = B_;
  const dim3 gv(grid_, B);
  const int rt = 32 * kRedTerms;
  k_density_sums<<<gv, kBlock, 0, stream>>>(r.a, red_);
  k_finish_sums<<<B, rt, 0, stream>>>(red_, grid_, red_out_);
  k_scale_factor<<<B, 32, 0, stream>>>(st_, red_out_, r.cc, p.dv, initial);
  k_rescale<<<gv, kBlock, 0, stream>>>(r.a, st_, r.cc, initial);
  r.eng->evaluate(r.a.rho, r.a.vext, r.mu_compute.data(), grad_, scalars_, stream);
  k_post_sums<<<gv, kBlock, 0, stream>>>(r.a, red_);
  k_finish_sums<<<B, rt, 0, stream>>>(red_, grid_, red_out_);
  k_post_control<<<B, 32, 0, stream>>>(st_, red_out_, r.cc);
  k_post_apply<<<gv, kBlock, 0, stream>>>(r.a, st_, r.cc, red_);
  k_finish_sums<<<B, rt, 0, stream>>>(red_, grid_, red_out_ + 4);
  if (r.cfg.mode == kSaddle) {
    k_project<<<gv, kBlock, 0, stream>>>(r.a, red_out_ + 4, red_);
    k_finish_sums<<<B, rt, 0, stream>>>(red_, grid_, red_out_ + 4);
  }
  k_fire_finalize<<<B, 32, 0, stream>>>(st_, red_out_ + 4, scalars_, r.cfg.fire, (double)N_, r.volume,
                                        r.cfg.use_monitor ? 1 : 0, initial);
}

void Drivers::fire_begin(const FireConfig& cfg, const double* mu, const double* mass, double* rho,
                         const double* direction, cudaStream_t stream, Engine* refine, double refine_switch) {
  const EvalParams& p = eng_.params();
  const int B = B_;
  if (!run_) run_.reset(new FireRun());
  FireRun& r = *run_;
  r = FireRun();
  r.cfg = cfg;
  Vec& a = r.a;
  a.x = x_;
  a.v = v_;
  a.f = f_;
  a.rho = rho;
  a.grad = grad_;
  a.dir = direction;
  a.vext = cfg.vext;
  a.N = N_;
  a.nx = p.nx;
  a.ny = p.ny;
  a.nz = p.nz;
  a.dv = p.dv;
  a.param = cfg.param;
  a.rho_min = cfg.rho_min;
  a.range = cfg.rho_max - cfg.rho_min;
  r.cc.mode = cfg.mode;
  r.cc.homogeneous = cfg.homogeneous_boundary ? 1 : 0;
  r.cc.boundary_mass = cfg.boundary_mass;
  const long long inner = (long long)std::max(p.nx - 2, 0) * std::max(p.ny - 2, 0) * std::max(p.nz - 2, 0);
  r.cc.n_face = (double)(N_ - inner);
  r.volume = (double)N_ * p.dv;
  // Minimizer::fixed_mass computes with mu = 0 (minimization.hpp:388); the
  // other modes with the given chemical potential.
  r.mu_compute.resize(B);
  r.mu_final.resize(B);
  for (int b = 0; b < B; ++b) {
    r.mu_final[b] = mu[b];
    r.mu_compute[b] = (cfg.mode == kFixedMass) ? 0.0 : mu[b];
  }
  r.eng = &eng_;
  r.refine = refine;
  r.refine_switch = refine_switch;
  reset_step_graph();  // a graph holds this run's arguments
  // initialise (fire.hpp:60-84)
  const FireParams& fp = cfg.fire;
  for (int b = 0; b < B; ++b) {
    FireDevState& s0 = st_host_[b];
    std::memset(&s0, 0, sizeof(s0));
    s0.dt = fp.dt;
    s0.alpha = fp.alpha_start;
    s0.vv = 1.0;
    s0.scale = 1.0;
    s0.active = 1;
    s0.target_mass = mass[b];
  }
  CDFT_CUDA(cudaMemcpyAsync(st_, st_host_, sizeof(FireDevState) * B, cudaMemcpyHostToDevice, stream));
  k_from_density<<<dim3(grid_, B), kBlock, 0, stream>>>(a, rho);
  fire_compute(1, stream);
  CDFT_CUDA(cudaGetLastError());
}

// one FIRE step (fire.hpp:86-165): the v and x updates, then compute
void Drivers::fire_launch_step(cudaStream_t stream) {
  FireRun& r = *run_;
  const int B = B_;
  const dim3 gv(grid_, B);
  const int rt = 32 * kRedTerms;
  k_power<<<gv, kBlock, 0, stream>>>(r.a, red_);
  k_finish_sums<<<B, rt, 0, stream>>>(red_, grid_, red_out_);
  k_fire_control1<<<B, 32, 0, stream>>>(st_, red_out_, r.cfg.fire);
  k_fire_vstep<<<gv, kBlock, 0, stream>>>(r.a, st_, red_);
  k_finish_sums<<<B, rt, 0, stream>>>(red_, grid_, red_out_);
  k_fire_ratio<<<B, 32, 0, stream>>>(st_, red_out_);
  k_fire_xstep<<<gv, kBlock, 0, stream>>>(r.a, st_);
  fire_compute(0, stream);
}

void Drivers::fire_read_state(cudaStream_t stream) {
  CDFT_CUDA(cudaMemcpyAsync(st_host_, st_, sizeof(FireDevState) * B_, cudaMemcpyDeviceToHost, stream));
}

int Drivers::fire_decide(cudaStream_t stream, bool* engine_changed) {
  FireRun& r = *run_;
  const FireParams& fp = r.cfg.fire;
  if (engine_changed) *engine_changed = false;
  if (r.done) return 0;
  bool any_active = false, all_close = true;
  double worst = 0.0;
  for (int b = 0; b < B_; ++b) {
    const FireDevState& h = st_host_[b];
    if (!h.active) continue;
    any_active = true;
    const double metric = r.cfg.use_monitor ? h.monitor : h.rms_force;
    worst = std::max(worst, metric);
    if (!(h.iteration > 0 && metric < r.refine_switch * fp.force_tolerance)) all_close = false;
  }
  if (r.refine && !r.refining && any_active && r.steps > 0) {
    if (r.best_metric == 0.0 || worst < 0.9 * r.best_metric) {
      r.best_metric = worst;
      r.stalled_checks = 0;
    } else if (++r.stalled_checks >= kStallChecks) {
      all_close = true;
    }
  }
  if (r.refine && !r.refining && all_close && r.steps < fp.max_steps) {
    // FP64 defect correction from here on: once every running problem is
    // within refine_switch of the tolerance, once the mixed-precision run
    // has stopped improving (its noise floor), or once all problems have
    // converged under the mixed-precision forces
    r.eng = r.refine;
    r.refining = true;
    if (engine_changed) *engine_changed = true;
    if (!any_active) {
      k_fire_reactivate<<<B_, 32, 0, stream>>>(st_, fp.max_steps);
      CDFT_CUDA(cudaGetLastError());
      any_active = true;
    }
  }
  if (!any_active || r.steps >= fp.max_steps) {
    r.done = true;
    return 0;
  }
  return std::max(1, std::min(r.cfg.check_interval, fp.max_steps - r.steps));
}

void Drivers::fire_advance(int steps) { run_->steps += steps; }

const Engine* Drivers::fire_engine() const { return run_ ? run_->eng : nullptr; }

std::vector<FireResult> Drivers::fire_finish(cudaStream_t stream) {
  FireRun& r = *run_;
  const int B = B_;
  std::vector<FireResult> out(B);
  bool any_uphill = false;
  for (int b = 0; b < B; ++b) {
    FireResult& o = out[b];
    o.iterations = st_host_[b].iteration;
    o.converged = st_host_[b].converged != 0;
    o.rms_force = st_host_[b].rms_force;
    o.uphill_error = st_host_[b].uphill_error != 0;
    any_uphill = any_uphill || o.uphill_error;
  }
  if (B == 1 && any_uphill) return out;
  // Final density (minimization.hpp:441-450, saddle_point.hpp:533-549): rho
  // already holds rho(x) with the mass rescale of the last compute, which is
  // exactly the reference's extraction from the final x.  The final total()
  // uses the caller's chemical potential (fixed mass iterates with mu = 0).
  r.eng->evaluate(r.a.rho, r.a.vext, r.mu_final.data(), grad_, scalars_, stream);
  std::vector<double> sc((size_t)B * kScalarCount);
  CDFT_CUDA(cudaMemcpyAsync(sc.data(), scalars_, sizeof(double) * sc.size(), cudaMemcpyDeviceToHost, stream));
  CDFT_CUDA(cudaStreamSynchronize(stream));
  for (int b = 0; b < B; ++b) {
    out[b].free_energy = sc[(size_t)b * kScalarCount + 0];
    out[b].grand_potential = sc[(size_t)b * kScalarCount + 1];
  }
  return out;
}

void Drivers::capture_step(cudaStream_t stream) {
  reset_step_graph();
  CDFT_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  try {
    fire_launch_step(stream);
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(stream, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  CDFT_CUDA(cudaStreamEndCapture(stream, &step_graph_));
  CDFT_CUDA(cudaGraphInstantiate(&step_exec_, step_graph_, 0));
  step_key_ = run_->eng;
}

std::vector<FireResult> Drivers::fire_loop(const FireConfig& cfg, const double* mu, const double* mass, double* rho,
                                           const double* direction, cudaStream_t stream, Engine* refine,
                                           double refine_switch, bool graphs) {
  fire_begin(cfg, mu, mass, rho, direction, stream, refine, refine_switch);
  for (;;) {
    fire_read_state(stream);
    CDFT_CUDA(cudaStreamSynchronize(stream));
    const int chunk = fire_decide(stream, nullptr);
    if (chunk == 0) break;
    // (re)capture the step for the engine now evaluating; every kernel
    // argument of a step is the same from one step to the next
    if (graphs && step_key_ != run_->eng) capture_step(stream);
    for (int k = 0; k < chunk; ++k) {
      if (graphs)
        CDFT_CUDA(cudaGraphLaunch(step_exec_, stream));
      else
        fire_launch_step(stream);
    }
    CDFT_CUDA(cudaGetLastError());
    fire_advance(chunk);
  }
  return fire_finish(stream);
}

std::vector<std::vector<FireResult>> fire_minimize_group(std::vector<GroupMember>& members, const FireConfig& cfg,
                                                         cudaStream_t stream) {
  if (members.empty()) return {};
  if (cfg.mode == kSaddle) throw Error(-1, "fire_minimize_group: the saddle mode is single-problem");
  const int M = (int)members.size();
  std::vector<std::vector<double>> masses(M);
  for (int m = 0; m < M; ++m) {
    GroupMember& g = members[m];
    if (!g.drivers || !g.mu || !g.rho) throw Error(-1, "fire_minimize_group: drivers, mu and rho are required");
    for (int k = 0; k < m; ++k)
      if (members[k].drivers == g.drivers) throw Error(-1, "fire_minimize_group: one member per engine");
    const int B = g.drivers->batch();
    masses[m].assign(B, 0.0);
    if (cfg.mode == kFixedMass) {
      if (!g.mass) throw Error(-1, "fire_minimize_group: fixed mass needs a target mass per problem");
      for (int b = 0; b < B; ++b) {
        if (!(g.mass[b] > 0.0)) throw Error(-1, "fire_minimize_group: target masses must be > 0");
        masses[m][b] = g.mass[b];
      }
    }
    if (g.refine && g.refine->batch() != B) throw Error(-1, "fire_minimize_group: refine engines need the same batch");
  }
  const bool graphs = step_graphs();
  // the group runs on its own stream, joined to the caller's at entry and exit
  cudaStream_t s0 = nullptr;
  CDFT_CUDA(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
  std::vector<cudaEvent_t> ev(M + 1, nullptr);
  for (cudaEvent_t& e : ev) CDFT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto release = [&] {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  };
  std::vector<std::vector<FireResult>> out(M);
  try {
    CDFT_CUDA(cudaEventRecord(ev[M], stream));
    CDFT_CUDA(cudaStreamWaitEvent(s0, ev[M], 0));
    for (int m = 0; m < M; ++m)
      members[m].drivers->fire_begin(cfg, members[m].mu, masses[m].data(), members[m].rho, nullptr, s0,
                                     members[m].refine, members[m].refine_switch);
    std::vector<std::pair<int, const Engine*>> key;
    for (;;) {
      for (int m = 0; m < M; ++m) members[m].drivers->fire_read_state(s0);
      CDFT_CUDA(cudaStreamSynchronize(s0));
      int chunk = 0;
      std::vector<int> running;
      for (int m = 0; m < M; ++m) {
        const int c = members[m].drivers->fire_decide(s0, nullptr);
        if (c > 0) {
          running.push_back(m);
          chunk = chunk ? std::min(chunk, c) : c;
        }
      }
      if (running.empty()) break;
      std::vector<std::pair<int, const Engine*>> now;
      for (int m : running) now.emplace_back(m, members[m].drivers->fire_engine());
      // one step of every running member on its own stream, forked from s0
      auto step = [&] {
        CDFT_CUDA(cudaEventRecord(ev[M], s0));
        for (int m : running) {
          cudaStream_t sm = members[m].drivers->graph_stream();
          CDFT_CUDA(cudaStreamWaitEvent(sm, ev[M], 0));
          members[m].drivers->fire_launch_step(sm);
          CDFT_CUDA(cudaEventRecord(ev[m], sm));
          CDFT_CUDA(cudaStreamWaitEvent(s0, ev[m], 0));
        }
      };
      if (graphs && (!exec || now != key)) {
        release();
        CDFT_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
        try {
          step();
        } catch (...) {
          cudaGraph_t g = nullptr;
          cudaStreamEndCapture(s0, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        CDFT_CUDA(cudaStreamEndCapture(s0, &graph));
        CDFT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        key = now;
      }
      for (int k = 0; k < chunk; ++k) {
        if (graphs)
          CDFT_CUDA(cudaGraphLaunch(exec, s0));
        else
          step();
      }
      CDFT_CUDA(cudaGetLastError());
      for (int m : running) members[m].drivers->fire_advance(chunk);
    }
    for (int m = 0; m < M; ++m) out[m] = members[m].drivers->fire_finish(s0);
  } catch (...) {
    cudaStreamSynchronize(s0);
    release();
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    cudaStreamDestroy(s0);
    throw;
  }
  CDFT_CUDA(cudaEventRecord(ev[M], s0));
  CDFT_CUDA(cudaStreamWaitEvent(stream, ev[M], 0));
  CDFT_CUDA(cudaStreamSynchronize(s0));
  release();
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  cudaStreamDestroy(s0);
  return out;
}

void Drivers::ensure_ddft() {
  if (ddft_ready_) return;
  const EvalParams& p = eng_.params();
  CDFT_CUDA(cudaMalloc(&ddft_k_, sizeof(double2) * 3 * p.Nk));
  CDFT_CUDA(cudaMalloc(&lam_, sizeof(double) * (p.nx + p.ny + p.nzh)));
  std::vector<double> lam(p.nx + p.ny + p.nzh);
  const double Dx = 1.0 / (p.dx * p.dx);
  for (int i = 0; i < p.nx; ++i) lam[i] = 2.0 * Dx * (std::cos(2.0 * kPi * i / p.nx) - 1.0);
  for (int i = 0; i < p.ny; ++i) lam[p.nx + i] = 2.0 * Dx * (std::cos(2.0 * kPi * i / p.ny) - 1.0);
  for (int i = 0; i < p.nzh; ++i) lam[p.nx + p.ny + i] = 2.0 * Dx * (std::cos(2.0 * kPi * i / p.nz) - 1.0);
  CDFT_CUDA(cudaMemcpy(lam_, lam.data(), sizeof(double) * lam.size(), cudaMemcpyHostToDevice));
  CDFT_CUFFT(cufftPlan3d(&plan_r2c_, p.nx, p.ny, p.nz, CUFFT_D2Z));
  CDFT_CUFFT(cufftPlan3d(&plan_c2r_, p.nx, p.ny, p.nz, CUFFT_Z2D));
  CDFT_CUDA(cudaMalloc(&ddft_st_, sizeof(DdftDevState)));
  CDFT_CUDA(cudaMallocHost(&ddft_st_host_, sizeof(DdftDevState)));
  std::memset(ddft_st_host_, 0, sizeof(DdftDevState));
  ddft_ready_ = true;
}

void Drivers::set_ddft_refine(Engine* refine, int iterations) {
  if (refine) {
    if (refine->precision() != kFP64) throw Error(-1, "ddft: the refine engine must be FP64");
    if (refine->points() != N_ || refine->species() != 1 || refine->batch() != 1)
      throw Error(-1, "ddft: the refine engine must have the driver's grid, one species and batch 1");
    if (iterations < 0) throw Error(-1, "ddft: refine iterations must be >= 0");
  }
  ddft_refine_ = refine;
  ddft_refine_iterations_ = refine ? iterations : 0;
}

// compute(rho0), R0_k and rho0_k (dynamics.hpp:347-354) from the step's
// copy of rho (v_), the iterate d1 (x_) <- rho, the control state reset.
void Drivers::ddft_prologue(const DDFTConfig& cfg, cudaStream_t s) {
  const EvalParams& p = eng_.params();
  CDFT_CUFFT(cufftSetStream(plan_r2c_, s));
  double2* rho0k = static_cast<double2*>(ddft_k_);
  double2* r0k = rho0k + p.Nk;
  const double mu = cfg.mu;
  eng_.evaluate(v_, nullptr, &mu, grad_, scalars_, s);
  k_ddft_rhs<<<grid_, kBlock, 0, s>>>(v_, grad_, tmp_, p.nx, p.ny, p.nz, p.dx, 1.0 / p.dv);
  CDFT_CUFFT(cufftExecD2Z(plan_r2c_, tmp_, r0k));
  CDFT_CUFFT(cufftExecD2Z(plan_r2c_, v_, rho0k));
  CDFT_CUDA(cudaMemcpyAsync(x_, v_, sizeof(double) * N_, cudaMemcpyDeviceToDevice, s));
  k_ddft_begin<<<1, 32, 0, s>>>(static_cast<DdftDevState*>(ddft_st_));
  CDFT_CUDA(cudaGetLastError());
}

// One fixed-point iteration (dynamics.hpp:362-389) and its decision.
void Drivers::ddft_body(const DDFTConfig& cfg, cudaStream_t s, unsigned long long cond, int use_cond) {
  const EvalParams& p = eng_.params();
  CDFT_CUFFT(cufftSetStream(plan_r2c_, s));
  CDFT_CUFFT(cufftSetStream(plan_c2r_, s));
  double2* rho0k = static_cast<double2*>(ddft_k_);
  double2* r0k = rho0k + p.Nk;
  double2* work = r0k + p.Nk;
  DdftDevState* st = static_cast<DdftDevState*>(ddft_st_);
  const double mu = cfg.mu;
  eng_.evaluate(x_, nullptr, &mu, grad_, scalars_, s);
  k_ddft_rhs<<<grid_, kBlock, 0, s>>>(x_, grad_, tmp_, p.nx, p.ny, p.nz, p.dx, 1.0 / p.dv);
  CDFT_CUFFT(cufftExecD2Z(plan_r2c_, tmp_, work));
  k_ddft_propagate<<<grid_, kBlock, 0, s>>>(rho0k, r0k, work, lam_, p.nx, p.ny, p.nzh, st);
  CDFT_CUFFT(cufftExecZ2D(plan_c2r_, work, tmp2_));
  k_ddft_update<<<grid_, kBlock, 0, s>>>(tmp2_, x_, N_, 1.0 / (double)N_, red_);
  k_maxmin_finish<<<1, 32, 0, s>>>(red_, grid_, red_out_);
  k_ddft_control<<<1, 32, 0, s>>>(st, red_out_, cfg.fp_tolerance, cfg.fp_max_iterations, kMaxRestarts,
                                  static_cast<cudaGraphConditionalHandle>(cond), use_cond);
  k_ddft_copy_back<<<grid_, kBlock, 0, s>>>(st, v_, x_, N_);
  CDFT_CUDA(cudaGetLastError());
}

// The FP64 refinement iterations (if any) and the final compute
// (dynamics.hpp:394).
void Drivers::ddft_epilogue(const DDFTConfig& cfg, cudaStream_t s) {
  const EvalParams& p = eng_.params();
  CDFT_CUFFT(cufftSetStream(plan_r2c_, s));
  CDFT_CUFFT(cufftSetStream(plan_c2r_, s));
  double2* rho0k = static_cast<double2*>(ddft_k_);
  double2* r0k = rho0k + p.Nk;
  double2* work = r0k + p.Nk;
  DdftDevState* st = static_cast<DdftDevState*>(ddft_st_);
  const double mu = cfg.mu;
  Engine& fin = ddft_refine_ ? *ddft_refine_ : eng_;
  for (int r = 0; r < ddft_refine_iterations_; ++r) {
    ddft_refine_->evaluate(x_, nullptr, &mu, grad_, scalars_, s);
    k_ddft_rhs<<<grid_, kBlock, 0, s>>>(x_, grad_, tmp_, p.nx, p.ny, p.nz, p.dx, 1.0 / p.dv);
    CDFT_CUFFT(cufftExecD2Z(plan_r2c_, tmp_, work));
    k_ddft_propagate<<<grid_, kBlock, 0, s>>>(rho0k, r0k, work, lam_, p.nx, p.ny, p.nzh, st);
    CDFT_CUFFT(cufftExecZ2D(plan_c2r_, work, tmp2_));
    k_ddft_update<<<grid_, kBlock, 0, s>>>(tmp2_, x_, N_, 1.0 / (double)N_, red_);
    k_maxmin_finish<<<1, 32, 0, s>>>(red_, grid_, red_out_);
    k_ddft_refine_record<<<1, 32, 0, s>>>(st, red_out_);
  }
  fin.evaluate(x_, nullptr, &mu, grad_, scalars_, s);
  CDFT_CUDA(cudaGetLastError());
}

// The whole step as one graph: the prologue, a conditional WHILE node whose
// body is one fixed-point iteration, the epilogue.  Each part is captured as
// an ordinary graph on the driver stream (the evaluation may fork its plane
// chunks onto other streams, which a capture straight into a conditional
// body does not support) and embedded as a child-graph node.
void Drivers::capture_ddft_step(const DDFTConfig& cfg) {
  reset_fp_graph();
  cudaStream_t s = graph_stream_;
  cudaGraph_t parts[3] = {nullptr, nullptr, nullptr};
  auto release_parts = [&] {
    for (cudaGraph_t& g : parts)
      if (g) cudaGraphDestroy(g);
  };
  auto capture = [&](int k, auto&& launches) {
    CDFT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      launches();
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    CDFT_CUDA(cudaStreamEndCapture(s, &parts[k]));
  };
  try {
    CDFT_CUDA(cudaGraphCreate(&fp_graph_, 0));
    cudaGraphConditionalHandle h = 0;
    CDFT_CUDA(cudaGraphConditionalHandleCreate(&h, fp_graph_, 1, cudaGraphCondAssignDefault));
    capture(0, [&] { ddft_prologue(cfg, s); });
    capture(1, [&] { ddft_body(cfg, s, h, 1); });
    capture(2, [&] { ddft_epilogue(cfg, s); });
    cudaGraphNode_t pro = nullptr, loop = nullptr, epi = nullptr, it = nullptr;
    CDFT_CUDA(cudaGraphAddChildGraphNode(&pro, fp_graph_, nullptr, 0, parts[0]));
    // zero-filled storage: the parameter union has no default constructor
    alignas(cudaGraphNodeParams) unsigned char np_buf[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(np_buf);
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    CDFT_CUDA(cudaGraphAddNode(&loop, fp_graph_, &pro, 1, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    CDFT_CUDA(cudaGraphAddChildGraphNode(&it, body, nullptr, 0, parts[1]));
    CDFT_CUDA(cudaGraphAddChildGraphNode(&epi, fp_graph_, &loop, 1, parts[2]));
    CDFT_CUDA(cudaGraphInstantiate(&fp_exec_, fp_graph_, 0));
  } catch (...) {
    release_parts();
    reset_fp_graph();
    throw;
  }
  release_parts();  // the child nodes hold copies
}

// integrating_factor_step (dynamics.hpp:333-401).  With step graphs on, the
// step runs on the driver's stream, joined to the caller's by events, as one
// graph launch; the host reads the control state and the energy once.
double Drivers::ddft_step(DDFTConfig& cfg, double* rho, cudaStream_t stream, int* fp_iterations) {
  ensure_ddft();
  const bool graphs = step_graphs() && !eng_.stage_timing_on() && !(ddft_refine_ && ddft_refine_->stage_timing_on());
  cudaStream_t s = stream;
  if (graphs) {
    ensure_graph_stream();
    CDFT_CUDA(cudaEventRecord(graph_ev_[0], stream));
    CDFT_CUDA(cudaStreamWaitEvent(graph_stream_, graph_ev_[0], 0));
    s = graph_stream_;
  }
  DdftDevState* hst = static_cast<DdftDevState*>(ddft_st_host_);
  try {
    hst->dt = cfg.dt;
    CDFT_CUDA(cudaMemcpyAsync(ddft_st_, hst, sizeof(double), cudaMemcpyHostToDevice, s));
    CDFT_CUDA(cudaMemcpyAsync(v_, rho, sizeof(double) * N_, cudaMemcpyDeviceToDevice, s));
    if (graphs) {
      DDFTGraphKey key;
      key.mu = cfg.mu;
      key.tol = cfg.fp_tolerance;
      key.min_density = cfg.min_density;
      key.diffusion = cfg.diffusion;
      key.fp_max = cfg.fp_max_iterations;
      key.refine_iterations = ddft_refine_iterations_;
      key.refine = ddft_refine_;
      key.gen = eng_.generation();
      key.refine_gen = ddft_refine_ ? ddft_refine_->generation() : 0;
      if (!fp_exec_ || !(key == fp_key_)) {
        capture_ddft_step(cfg);
        fp_key_ = key;
      }
      CDFT_CUDA(cudaGraphLaunch(fp_exec_, s));
    } else {
      ddft_prologue(cfg, s);
      // the same kernels, the host reading the decision after every iteration
      for (int guard = 0; guard < (kMaxRestarts + 1) * std::max(cfg.fp_max_iterations, 1); ++guard) {
        ddft_body(cfg, s, 0, 0);
        CDFT_CUDA(cudaMemcpyAsync(hst, ddft_st_, sizeof(DdftDevState), cudaMemcpyDeviceToHost, s));
        CDFT_CUDA(cudaStreamSynchronize(s));
        if (hst->status != 0) break;
      }
      ddft_epilogue(cfg, s);
    }
    CDFT_CUDA(cudaMemcpyAsync(rho, x_, sizeof(double) * N_, cudaMemcpyDeviceToDevice, s));
    CDFT_CUDA(cudaMemcpyAsync(hst, ddft_st_, sizeof(DdftDevState), cudaMemcpyDeviceToHost, s));
    CDFT_CUDA(cudaMemcpyAsync(host_pin_, scalars_, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
    CDFT_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    if (graphs) {
      reset_fp_graph();
      cudaEventRecord(graph_ev_[1], graph_stream_);
      cudaStreamWaitEvent(stream, graph_ev_[1], 0);
    }
    throw;
  }
  if (graphs) {
    CDFT_CUDA(cudaEventRecord(graph_ev_[1], graph_stream_));
    CDFT_CUDA(cudaStreamWaitEvent(stream, graph_ev_[1], 0));
  }
  cfg.dt = hst->dt;
  ddft_info_.fp_iterations = hst->total_it;
  ddft_info_.restarts = hst->restarts;
  ddft_info_.status = hst->status;
  ddft_info_.device_loop = graphs ? 1 : 0;
  ddft_info_.refine_deviation = hst->refine_deviation;
  if (fp_iterations) *fp_iterations = hst->total_it;
  return host_pin_[1];
}

}  // namespace cdft

namespace cdft {

Drivers::EigenResult Drivers::eigen_solve(const EigenConfig& cfg, const double* rho, double mu, double* vec,
                                          bool use_guess, cudaStream_t stream, Engine* hvp_engine) {
  if (cfg.method == kLanczos) {
    if (!cfg.exact_hvp) throw Error(-1, "eigen: the Lanczos solver needs exact products (exact_hvp = 1)");
    Engine& he = hvp_engine ? *hvp_engine : eng_;
    if (he.points() != N_ || he.species() != 1)
      throw Error(-1, "eigen: the product engine must have the driver's grid and one species");
    LanczosConfig lc;
    lc.tolerance = cfg.tolerance;
    lc.max_iterations = cfg.max_iterations;
    lc.block = cfg.block;
    lc.max_basis = cfg.max_basis;
    lc.check_interval = cfg.check_interval;
    lc.seed = cfg.seed;
    const LanczosResult lr = lanczos_lowest(he, lc, rho, vec, use_guess, stream);
    EigenResult r;
    r.eigenvalue = lr.eigenvalue;
    r.iterations = lr.iterations;
    r.converged = lr.converged;
    (void)mu;  // the Hessian does not depend on mu
    return r;
  }
  if (cfg.method != kRayleighRitz) throw Error(-1, "eigen: unknown method");
  for (double*& p : ev_)
    if (!p) CDFT_CUDA(cudaMalloc(&p, sizeof(double) * N_));
  double* f0 = ev_[0];
  double* hv = ev_[1];
  double* q1 = ev_[2];
  double* hq1 = ev_[3];
  double* q2 = ev_[4];
  double* hq2 = ev_[5];
  double* praw = ev_[6];
  double* vnew = ev_[7];
  double* v = vec;
  force(rho, f0, mu, 1, stream);
  auto H = [&](const double* in, double* out) {
    if (cfg.exact_hvp)
      hvp_exact(rho, in, out, mu, 1, stream);
    else
      hvp_fd(rho, f0, in, out, cfg.hessian_eps, mu, 1, stream);
  };
  if (!use_guess) k_randn<<<grid_, kBlock, 0, stream>>>(v, N_, cfg.seed);
  {
    const double nv = std::sqrt(dot(v, v, N_, stream));
    axpby(0.0, v, 1.0 / nv, v, N_, stream);
  }
  H(v, hv);
  double lambda = dot(v, hv, N_, stream);
  bool have_p = false;
  EigenResult res;
  int iter = 0;
  for (; iter < cfg.max_iterations; ++iter) {
    // residual = hv - lambda v (into q1)
    k_lincomb<<<grid_, kBlock, 0, stream>>>(q1, 1.0, hv, -lambda, v, 0.0, nullptr, N_);
    const double rn = std::sqrt(dot(q1, q1, N_, stream));
    if (rn < cfg.tolerance) {
      res.converged = true;
      break;
    }
    const double rq = dot(q1, v, N_, stream);
    axpby(-rq, v, 1.0, q1, N_, stream);
    const double q1n = std::sqrt(dot(q1, q1, N_, stream));
    if (q1n < 1e-30) break;
    axpby(0.0, q1, 1.0 / q1n, q1, N_, stream);
    H(q1, hq1);
    int dim = 2;
    if (have_p) {
      const double a0 = dot(praw, v, N_, stream);
      const double a1 = dot(praw, q1, N_, stream);
      k_lincomb<<<grid_, kBlock, 0, stream>>>(q2, 1.0, praw, -a0, v, -a1, q1, N_);
      const double q2n = std::sqrt(dot(q2, q2, N_, stream));
      if (q2n > 1e-10) {
        axpby(0.0, q2, 1.0 / q2n, q2, N_, stream);
        H(q2, hq2);
        dim = 3;
      }
    }
    double Hm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    Hm[0][0] = dot(v, hv, N_, stream);
    Hm[0][1] = Hm[1][0] = dot(v, hq1, N_, stream);
    Hm[1][1] = dot(q1, hq1, N_, stream);
    if (dim == 3) {
      Hm[0][2] = Hm[2][0] = dot(v, hq2, N_, stream);
      Hm[1][2] = Hm[2][1] = dot(q1, hq2, N_, stream);
      Hm[2][2] = dot(q2, hq2, N_, stream);
    }
    double c[3] = {0, 0, 0}, ev = 0.0;
    smallest_eigvec(dim, Hm, c, &ev);
    k_lincomb<<<grid_, kBlock, 0, stream>>>(vnew, c[0], v, c[1], q1, dim == 3 ? c[2] : 0.0,
                                            dim == 3 ? q2 : nullptr, N_);
    k_lincomb<<<grid_, kBlock, 0, stream>>>(praw, 1.0, vnew, -1.0, v, 0.0, nullptr, N_);
    have_p = true;
    const double nn = std::sqrt(dot(vnew, vnew, N_, stream));
    k_lincomb<<<grid_, kBlock, 0, stream>>>(v, 1.0 / nn, vnew, 0.0, nullptr, 0.0, nullptr, N_);
    H(v, hv);
    lambda = dot(v, hv, N_, stream);
  }
  res.eigenvalue = lambda;
  res.iterations = iter;
  return res;
}

Drivers::SaddleResult Drivers::saddle_find(const SaddleConfig& cfg, double* rho, double mu, double target_mass,
                                           double* eigvec, cudaStream_t stream, Engine* refine, Engine* hvp_engine,
                                           double refine_switch) {
  const EvalParams& p = eng_.params();
  double* dir = nullptr;
  CDFT_CUDA(cudaMalloc(&dir, sizeof(double) * N_));
  SaddleResult res;
  double omega = 0.0;
  double ftol = cfg.tolerance_start;
  bool have_vec = false;
  int outer = 0;
  try {
    for (; outer < cfg.max_outer_iterations; ++outer) {
      const double omega_old = omega;
      const bool guess = have_vec && outer >= cfg.eigenvalue_clear_count;
      EigenConfig ec = cfg.eigen;
      ec.seed = cfg.eigen.seed + (unsigned long long)outer;
      EigenResult er = eigen_solve(ec, rho, mu, eigvec, guess, stream, hvp_engine);
      have_vec = true;
      res.eigenvalue = er.eigenvalue;
      res.eigen_iterations += er.iterations;
      // direction in parameter space, normalised (saddle_point.hpp:424-430)
      k_dir_alias<<<grid_, kBlock, 0, stream>>>(eigvec, rho, dir, N_, cfg.rho_min);
      const double dn = std::sqrt(dot(dir, dir, N_, stream));
      if (dn > 1e-30) axpby(0.0, dir, 1.0 / dn, dir, N_, stream);
      // boundary mass (saddle_point.hpp:432-443)
      k_face_sum<<<grid_, kBlock, 0, stream>>>(rho, N_, p.nx, p.ny, p.nz, red_);
      k_finish_sums<<<1, 32 * kRedTerms, 0, stream>>>(red_, grid_, red_out_);
      CDFT_CUDA(cudaMemcpyAsync(host_pin_, red_out_, sizeof(double), cudaMemcpyDeviceToHost, stream));
      CDFT_CUDA(cudaStreamSynchronize(stream));
      const long long inner = (long long)std::max(p.nx - 2, 0) * std::max(p.ny - 2, 0) * std::max(p.nz - 2, 0);
      const double n_face = (double)(N_ - inner);
      const double avg = n_face > 0 ? host_pin_[0] / n_face : 0.0;
      FireConfig fc;
      fc.fire = cfg.fire;
      fc.fire.force_tolerance = std::max(ftol, cfg.fire.force_tolerance);
      ftol /= cfg.tolerance_factor;
      fc.mode = kSaddle;
      fc.param = kUnbounded;
      fc.rho_min = cfg.rho_min;
      fc.homogeneous_boundary = false;
      fc.mu = mu;
      fc.target_mass = target_mass;
      fc.boundary_mass = avg * p.dv * n_face;
      fc.use_monitor = false;
      FireResult fr = fire_minimize(fc, rho, dir, stream, refine, refine_switch);
      if (fr.uphill_error) throw Error(-2, "fire::step: exceeded max uphill steps");
      omega = fr.grand_potential;
      res.fire_steps += fr.iterations;
      if (outer > 0 && std::abs(omega - omega_old) < cfg.omega_tolerance) {
        res.converged = true;
        break;
      }
    }
  } catch (...) {
    cudaFree(dir);
    throw;
  }
  cudaFree(dir);
  res.grand_potential = omega;
  res.outer_iterations = outer + 1;  // as the reference reports it (saddle_point.hpp:584)
  return res;
}

// ---------------------------------------------------- split / CN / run

double Drivers::ddft_split_step(const DDFTConfig& cfg, double* rho, cudaStream_t stream) {
  ensure_ddft();
  const EvalParams& p = eng_.params();
  CDFT_CUFFT(cufftSetStream(plan_r2c_, stream));
  CDFT_CUFFT(cufftSetStream(plan_c2r_, stream));
  double2* work = static_cast<double2*>(ddft_k_);
  const double inv_n = 1.0 / (double)N_;
  double* star = x_;   // rho*, then rho**
  double* f = grad_;
  double* rhs = tmp_;
  // half diffusion (dynamics.hpp:423-437)
  CDFT_CUFFT(cufftExecD2Z(plan_r2c_, rho, work));
  k_half_diffusion<<<grid_, kBlock, 0, stream>>>(work, p.nx, p.ny, p.nzh, p.nz, p.dx, cfg.diffusion, cfg.dt);
  CDFT_CUFFT(cufftExecZ2D(plan_c2r_, work, tmp2_));
  k_scale_clamp<<<grid_, kBlock, 0, stream>>>(tmp2_, nullptr, star, N_, inv_n, 0.0, cfg.min_density);
  // forward-Euler excess step (dynamics.hpp:439-443)
  eng_.evaluate(star, nullptr, &cfg.mu, f, scalars_, stream);
  k_ddft_rhs<<<grid_, kBlock, 0, stream>>>(star, f, rhs, p.nx, p.ny, p.nz, p.dx, 1.0 / p.dv);
  k_scale_clamp<<<grid_, kBlock, 0, stream>>>(star, rhs, star, N_, 1.0, cfg.dt, cfg.min_density);
  // half diffusion (dynamics.hpp:445-456)
  CDFT_CUFFT(cufftExecD2Z(plan_r2c_, star, work));
  k_half_diffusion<<<grid_, kBlock, 0, stream>>>(work, p.nx, p.ny, p.nzh, p.nz, p.dx, cfg.diffusion, cfg.dt);
  CDFT_CUFFT(cufftExecZ2D(plan_c2r_, work, tmp2_));
  k_scale_clamp<<<grid_, kBlock, 0, stream>>>(tmp2_, nullptr, rho, N_, inv_n, 0.0, cfg.min_density);
  CDFT_CUDA(cudaGetLastError());
  return force(rho, f, cfg.mu, 0, stream);  // the energy of the final state (dynamics.hpp:458)
}

double Drivers::ddft_cn_step(const DDFTConfig& cfg, double* rho, cudaStream_t stream, int* fp_iterations) {
  ensure_ddft();
  const EvalParams& p = eng_.params();
  CDFT_CUFFT(cufftSetStream(plan_r2c_, stream));
  CDFT_CUFFT(cufftSetStream(plan_c2r_, stream));
  double2* rho0k = static_cast<double2*>(ddft_k_);
  double2* r0k = rho0k + p.Nk;
  double2* work = r0k + p.Nk;
  double* d1 = x_;
  double* f = grad_;
  double* rhs = tmp_;
  const double inv_n = 1.0 / (double)N_;
  // rho0_k, R0_k (dynamics.hpp:491-500)
  CDFT_CUFFT(cufftExecD2Z(plan_r2c_, rho, rho0k));
  eng_.evaluate(rho, nullptr, &cfg.mu, f, scalars_, stream);
  k_ddft_rhs<<<grid_, kBlock, 0, stream>>>(rho, f, rhs, p.nx, p.ny, p.nz, p.dx, 1.0 / p.dv);
  CDFT_CUFFT(cufftExecD2Z(plan_r2c_, rhs, r0k));
  CDFT_CUDA(cudaMemcpyAsync(d1, rho, sizeof(double) * N_, cudaMemcpyDeviceToDevice, stream));
  int it = 0;
  for (; it < cfg.fp_max_iterations; ++it) {  // dynamics.hpp:505-530
    eng_.evaluate(d1, nullptr, &cfg.mu, f, scalars_, stream);
    k_ddft_rhs<<<grid_, kBlock, 0, stream>>>(d1, f, rhs, p.nx, p.ny, p.nz, p.dx, 1.0 / p.dv);
    CDFT_CUFFT(cufftExecD2Z(plan_r2c_, rhs, work));
    k_cn_combine<<<grid_, kBlock, 0, stream>>>(rho0k, r0k, work, p.nx, p.ny, p.nzh, p.nz, p.dx, cfg.diffusion,
                                               cfg.dt);
    CDFT_CUFFT(cufftExecZ2D(plan_c2r_, work, tmp2_));
    k_cn_update<<<grid_, kBlock, 0, stream>>>(tmp2_, d1, N_, inv_n, cfg.min_density, red_);
    k_maxmin_finish<<<1, 32, 0, stream>>>(red_, grid_, red_out_);
    CDFT_CUDA(cudaMemcpyAsync(host_pin_, red_out_, sizeof(double), cudaMemcpyDeviceToHost, stream));
    CDFT_CUDA(cudaStreamSynchronize(stream));
    if (host_pin_[0] < cfg.fp_tolerance) {
      ++it;
      break;
    }
  }
  if (fp_iterations) *fp_iterations = it;
  CDFT_CUDA(cudaMemcpyAsync(rho, d1, sizeof(double) * N_, cudaMemcpyDeviceToDevice, stream));
  return force(rho, f, cfg.mu, 0, stream);  // dynamics.hpp:532
}

int Drivers::ddft_run(DDFTConfig& cfg, int n_steps, double* rho, double* times, double* energies,
                      int snapshot_interval, SnapshotSink* snaps, StopFn stop, void* user, const Reservoir* reservoir,
                      cudaStream_t stream) {
  const bool res = reservoir && reservoir->mask;
  auto apply_boundary = [&]() {
    if (res) k_reservoir_fill<<<grid_, kBlock, 0, stream>>>(rho, reservoir->mask, N_, reservoir->density);
  };
  const bool snapping = snaps && snaps->host && snapshot_interval > 0 && snaps->capacity > 0;
  if (snapping && !copy_stream_) {
    CDFT_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      CDFT_CUDA(cudaMalloc(&snap_stage_[i], sizeof(double) * N_));
      CDFT_CUDA(cudaEventCreateWithFlags(&snap_ready_[i], cudaEventDisableTiming));
      CDFT_CUDA(cudaEventCreateWithFlags(&snap_done_[i], cudaEventDisableTiming));
    }
  }
  if (snaps) snaps->count = 0;
  int issued = 0;
  // the snapshot of the current density: a device copy into a staging
  // buffer on the compute stream, then its D2H copy on the copy stream, so
  // the next steps run while it drains
  auto snapshot = [&](int step) {
    if (!snapping || snaps->count >= snaps->capacity) return;
    const int k = issued & 1;
    if (issued >= 2) CDFT_CUDA(cudaStreamWaitEvent(stream, snap_done_[k], 0));
    CDFT_CUDA(cudaMemcpyAsync(snap_stage_[k], rho, sizeof(double) * N_, cudaMemcpyDeviceToDevice, stream));
    CDFT_CUDA(cudaEventRecord(snap_ready_[k], stream));
    CDFT_CUDA(cudaStreamWaitEvent(copy_stream_, snap_ready_[k], 0));
    CDFT_CUDA(cudaMemcpyAsync(snaps->host + (size_t)snaps->count * N_, snap_stage_[k], sizeof(double) * N_,
                              cudaMemcpyDeviceToHost, copy_stream_));
    CDFT_CUDA(cudaEventRecord(snap_done_[k], copy_stream_));
    if (snaps->steps) snaps->steps[snaps->count] = step;
    ++snaps->count;
    ++issued;
  };
  // Simulation::run (dynamics.hpp:597-649): initial energy, then steps with
  // the adaptive time step
  apply_boundary();
  // the initial energy from the FP64 refine engine when there is one, as
  // every step's final energy
  double e0 = 0.0;
  if (ddft_refine_) {
    ddft_refine_->evaluate(rho, nullptr, &cfg.mu, tmp2_, scalars_, stream);
    CDFT_CUDA(cudaMemcpyAsync(host_pin_, scalars_, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
    CDFT_CUDA(cudaStreamSynchronize(stream));
    e0 = host_pin_[1];
  } else {
    e0 = force(rho, tmp2_, cfg.mu, 0, stream);
  }
  if (times) times[0] = 0.0;
  if (energies) energies[0] = e0;
  snapshot(0);
  int successes = 0, step = 1;
  double time = 0.0;
  for (; step <= n_steps; ++step) {
    const double dt_before = cfg.dt;
    const double e = ddft_step(cfg, rho, stream, nullptr);
    const double dt_used = cfg.dt;
    time += dt_used;
    apply_boundary();
    if (dt_used < dt_before)
      successes = 0;
    else
      ++successes;
    if (successes >= 5 && cfg.dt < cfg.dt_max) {
      cfg.dt = std::min(2.0 * cfg.dt, cfg.dt_max);
      successes = 0;
    }
    if (times) times[step] = time;
    if (energies) energies[step] = e;
    if (snapshot_interval > 0 && step % snapshot_interval == 0) snapshot(step);
    if (stop && stop(step, time, e, user)) {
      ++step;
      break;
    }
  }
  if (snapping) CDFT_CUDA(cudaStreamSynchronize(copy_stream_));
  return step - 1;
}

// ------------------------------------------------------------------ Picard

std::vector<Drivers::PicardResult> Drivers::picard(const PicardConfig& cfg, const double* mu, const double* mass,
                                                   const double* background, double* rho, cudaStream_t stream) {
  const EvalParams& p = eng_.params();
  const int B = B_;
  if (!(cfg.mixing > 0.0) || cfg.max_iterations < 0) throw Error(-1, "picard: mixing > 0 and max_iterations >= 0");
  std::vector<double> muv(mu, mu + B);
  PicardDevState* st = reinterpret_cast<PicardDevState*>(st_);  // the FIRE state slots (larger) hold it
  static_assert(sizeof(PicardDevState) <= sizeof(FireDevState), "state slot");
  std::vector<PicardDevState> h(B);
  for (int b = 0; b < B; ++b) {
    h[b] = PicardDevState{};
    h[b].active = 1;
    h[b].scale = 1.0;
    h[b].target_mass = mass ? mass[b] : 0.0;
  }
  CDFT_CUDA(cudaMemcpyAsync(st, h.data(), sizeof(PicardDevState) * B, cudaMemcpyHostToDevice, stream));
  const dim3 gv(grid_, B);
  const int rt = 32 * kRedTerms;
  const double n_dof = (double)N_;
  int steps = 0;
  auto all_done = [&]() {
    CDFT_CUDA(cudaMemcpyAsync(h.data(), st, sizeof(PicardDevState) * B, cudaMemcpyDeviceToHost, stream));
    CDFT_CUDA(cudaStreamSynchronize(stream));
    for (const auto& x : h)
      if (x.active) return false;
    return true;
  };
  while (steps < cfg.max_iterations && !all_done()) {
    const int chunk = std::max(1, std::min(cfg.check_interval, cfg.max_iterations - steps));
    for (int k = 0; k < chunk; ++k) {
      eng_.evaluate(rho, nullptr, muv.data(), grad_, scalars_, stream);
      k_sum_sq<<<gv, kBlock, 0, stream>>>(grad_, N_, red_);
      k_finish_sums<<<B, rt, 0, stream>>>(red_, grid_, red_out_);
      k_picard_control<<<B, 32, 0, stream>>>(st, red_out_, scalars_, n_dof, cfg.tolerance);
      k_picard_update<<<gv, kBlock, 0, stream>>>(rho, grad_, st, N_, cfg.mixing / p.dv, cfg.min_density);
      if (mass) {
        k_excess_sum<<<gv, kBlock, 0, stream>>>(rho, background, N_, red_);
        k_finish_sums<<<B, rt, 0, stream>>>(red_, grid_, red_out_);
        k_picard_mass<<<B, 32, 0, stream>>>(st, red_out_, p.dv);
        k_picard_rescale<<<gv, kBlock, 0, stream>>>(rho, background, st, N_, cfg.constraint_min_density);
      }
      k_picard_count<<<B, 32, 0, stream>>>(st);
    }
    CDFT_CUDA(cudaGetLastError());
    steps += chunk;
  }
  all_done();  // the state after the last chunk
  std::vector<PicardResult> out(B);
  for (int b = 0; b < B; ++b) {
    const PicardDevState& x = h[b];
    out[b].grand_potential = x.omega;
    out[b].residual = x.residual;
    out[b].iterations = x.iter;
    // picard.hpp:121: the converged flag after the loop, with omega_prev as
    // the loop left it (equal to omega when max_iterations ran out)
    out[b].converged = x.converged || x.residual < cfg.tolerance ||
                       (x.iter > 0 && std::fabs(x.omega - x.omega_prev) < cfg.tolerance);
  }
  return out;
}

}  // namespace cdft
