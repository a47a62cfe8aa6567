// The pair-potential pieces and the mean-field cell weight as inline
// functions for both the host set-up code (physics.cpp) and the device-side
// weight kernel (engine.cu): potentials.hpp:71-236 (raw potentials, the
// WCA / Barker-Henderson split) and mean_field.hpp:42-134 (cell weights).
#pragma once

#include <cmath>

#include "physics.hpp"

#ifdef __CUDACC__
#define CDFT_PHD __host__ __device__ inline
#else
#define CDFT_PHD inline
#endif

namespace cdft {
namespace phys {

constexpr double kMaxPotential = 1e50;

// V(r) before shifting (potentials.hpp:71-75, 135-143, 199-206).
CDFT_PHD double raw_potential(const Potential& p, double r) {
  if (p.type == kLennardJones) {
    const double y = p.sigma / r;
    const double y6 = y * y * y * y * y * y;
    return 4.0 * p.epsilon * (y6 * y6 - y6);
  }
  if (p.type == kTenWoldeFrenkel) {
    if (r < p.sigma) return kMaxPotential;
    const double s = r / p.sigma;
    const double y = 1.0 / (s * s - 1.0);
    const double y3 = y * y * y;
    return (4.0 * p.epsilon / (p.alpha * p.alpha)) * (y3 * y3 - p.alpha * y3);
  }
  // WRDF: epsilon_shift holds eps_eff
  if (r >= p.r_cutoff) return 0.0;
  const double y = p.sigma / r;
  const double z = p.r_cutoff / r;
  return p.epsilon_shift * (y * y - 1.0) * (z * z - 1.0) * (z * z - 1.0);
}

CDFT_PHD double split_point(const Potential& p, int split) {
  if (p.type == kWRDF) return p.r_min;
  return split == kBarkerHenderson ? p.r_zero : p.r_min;
}

// potentials.hpp:88-94, 157-163, 221-226
CDFT_PHD double repulsive(const Potential& p, double r, int split) {
  if (p.type == kWRDF) {
    if (split == kBarkerHenderson) return (r < p.r_min) ? phys::raw_potential(p, r) : 0.0;
    return (r < p.r_min) ? phys::raw_potential(p, r) - p.v_min : 0.0;
  }
  const double v = phys::raw_potential(p, r) - p.epsilon_shift;
  if (split == kBarkerHenderson) return (r < p.r_zero) ? v : 0.0;
  return (r < p.r_min) ? v - p.v_min : 0.0;
}

// potentials.hpp:97-107, 165-175, 228-236
CDFT_PHD double attractive(const Potential& p, double r, int split) {
  if (p.type == kWRDF) {
    if (r >= p.r_cutoff) return 0.0;
    if (split == kBarkerHenderson) return (r >= p.r_min) ? phys::raw_potential(p, r) : 0.0;
    return (r >= p.r_min) ? phys::raw_potential(p, r) : p.v_min;
  }
  const double rc = p.r_cutoff > 0.0 ? p.r_cutoff : 1e30;
  if (r >= rc) return 0.0;
  const double v = phys::raw_potential(p, r) - p.epsilon_shift;
  if (split == kBarkerHenderson) return (r >= p.r_zero) ? v : 0.0;
  return (r >= p.r_min) ? v : p.v_min;
}

// mean_field.hpp:42-134: the weight of the cell at offset (sx, sy, sz).
CDFT_PHD double cell_weight(const Potential& p, int split, int scheme, double kT, double dx, long sx, long sy,
                            long sz) {
  if (scheme == kWeightZero) {
    const double r2 = static_cast<double>(sx * sx + sy * sy + sz * sz) * dx * dx;
    return phys::attractive(p, std::sqrt(r2), split) / kT;
  }
  if (scheme == kWeightQuadraticF) {
    // 27-point tensor rule: nodes -1/2, 0, 1/2 of the cell, weights 1/3 each
    const double third = 1.0 / 3.0;
    double sum = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) {
          const double rx = (static_cast<double>(sx) + 0.5 * (i - 1)) * dx;
          const double ry = (static_cast<double>(sy) + 0.5 * (j - 1)) * dx;
          const double rz = (static_cast<double>(sz) + 0.5 * (k - 1)) * dx;
          const double r = std::sqrt(rx * rx + ry * ry + rz * rz);
          sum += third * third * third * phys::attractive(p, r, split) / kT;
        }
    return sum;
  }
  // linear (E/F) and the Gauss schemes share the 8-corner average
  double sum = 0.0;
  for (int di = 0; di <= 1; ++di)
    for (int dj = 0; dj <= 1; ++dj)
      for (int dk = 0; dk <= 1; ++dk) {
        const double x = (static_cast<double>(sx) - 0.5 + static_cast<double>(di)) * dx;
        const double y = (static_cast<double>(sy) - 0.5 + static_cast<double>(dj)) * dx;
        const double z = (static_cast<double>(sz) - 0.5 + static_cast<double>(dk)) * dx;
        const double r = std::sqrt(x * x + y * y + z * z);
        sum += phys::attractive(p, r, split) / kT;
      }
  return sum / 8.0;
}

// mean_field.hpp:160-185: the signed offset of grid index i on an axis of n
// points, and whether a cell lies beyond the cut-off plus half a cell
// diagonal (its weight is then zero without evaluation).
CDFT_PHD long signed_offset(long i, long n) { return (i <= n / 2) ? i : i - n; }

CDFT_PHD bool cell_skipped(const Potential& p, double dx, long sx, long sy, long sz) {
  if (!(p.r_cutoff > 0.0)) return false;
  const double r_skip = p.r_cutoff + std::sqrt(3.0) * 0.5 * dx;
  const double dist2 = static_cast<double>(sx * sx + sy * sy + sz * sz) * dx * dx;
  return dist2 > r_skip * r_skip;
}

}  // namespace phys
}  // namespace cdft
