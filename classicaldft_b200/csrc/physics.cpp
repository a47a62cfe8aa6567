// Set-up physics on the host: pair potentials with their WCA / Barker-Henderson
// split, the hard-sphere diameter and van der Waals integrals, and the
// real-space mean-field cell weights.  This is one-off set-up work per grid and
// temperature (include/dft/physics/potentials.hpp, functionals/mean_field.hpp:42-196);
// the evaluation itself runs on the GPU.
#include "physics.hpp"

#include "physics_fn.cuh"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <vector>

namespace cdft {

namespace {
constexpr double kPiD = 3.14159265358979323846;
constexpr double kMaxPotential = 1e50;
}  // namespace

// potentials.hpp:311-368 (factories)
Potential make_potential(int type, double sigma, double epsilon, double r_cutoff, double alpha) {
  Potential p;
  p.type = type;
  p.sigma = sigma;
  p.epsilon = epsilon;
  p.r_cutoff = r_cutoff;
  p.alpha = alpha;
  if (type == kLennardJones) {
    auto vr = [&](double r) {
      double y = sigma / r;
      double y6 = y * y * y * y * y * y;
      return 4.0 * epsilon * (y6 * y6 - y6);
    };
    p.epsilon_shift = (r_cutoff > 0.0) ? vr(r_cutoff) : 0.0;
    p.r_min = std::pow(2.0, 1.0 / 6.0) * sigma;
    p.v_min = vr(p.r_min) - p.epsilon_shift;
    p.r_zero = sigma * std::pow(0.5 * std::sqrt(1.0 + p.epsilon_shift / epsilon) + 0.5, -1.0 / 6.0);
  } else if (type == kTenWoldeFrenkel) {
    auto vr = [&](double r) -> double {
      if (r < sigma) return kMaxPotential;
      double s = r / sigma;
      double y = 1.0 / (s * s - 1.0);
      double y3 = y * y * y;
      return (4.0 * epsilon / (alpha * alpha)) * (y3 * y3 - alpha * y3);
    };
    p.epsilon_shift = (r_cutoff > 0.0) ? vr(r_cutoff) : 0.0;
    p.r_min = sigma * std::sqrt(1.0 + std::pow(2.0 / alpha, 1.0 / 3.0));
    p.v_min = vr(p.r_min) - p.epsilon_shift;
    p.r_zero = sigma * std::sqrt(1.0 + std::pow(25.0 * std::sqrt(1.0 + p.epsilon_shift) + 25.0, -1.0 / 3.0));
  } else if (type == kWRDF) {
    double rc_s = r_cutoff / sigma;
    p.epsilon_shift = epsilon * 2.0 * rc_s * rc_s * std::pow(2.0 * (rc_s * rc_s - 1.0) / 3.0, -3.0);  // eps_eff
    p.r_min = r_cutoff * std::pow((1.0 + 2.0 * rc_s * rc_s) / 3.0, -0.5);
    p.v_min = raw_potential(p, p.r_min);
    p.r_zero = p.r_min;
  } else {
    throw std::invalid_argument("unknown potential type");
  }
  return p;
}

// The potential pieces live in physics_fn.cuh, shared with the device.
double raw_potential(const Potential& p, double r) { return phys::raw_potential(p, r); }
double split_point(const Potential& p, int split) { return phys::split_point(p, split); }
double hard_core(const Potential& p) { return p.type == kTenWoldeFrenkel ? p.sigma : 0.0; }
double repulsive(const Potential& p, double r, int split) { return phys::repulsive(p, r, split); }
double attractive(const Potential& p, double r, int split) { return phys::attractive(p, r, split); }

// ------------------------------------------------------------ quadrature

namespace {

struct GaussRule {
  std::vector<double> x, w;
};

// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_n.
GaussRule gauss_legendre(int n) {
  GaussRule g;
  g.x.resize(n);
  g.w.resize(n);
  for (int i = 0; i < n; ++i) {
    double x = std::cos(kPiD * (i + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (x * p1 - p0) / (x * x - 1.0);
      double dx = p1 / dp;
      x -= dx;
      if (std::abs(dx) < 1e-16) break;
    }
    g.x[i] = x;
    g.w[i] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
  return g;
}

template <class F>
double rule(const GaussRule& g, F&& f, double a, double b) {
  double c = 0.5 * (a + b), h = 0.5 * (b - a), s = 0.0;
  for (size_t i = 0; i < g.x.size(); ++i) s += g.w[i] * f(c + h * g.x[i]);
  return s * h;
}

}  // namespace

// Globally adaptive bisection with a 10/21-point Gauss-Legendre error
// estimate; plays the role of GSL QAGS (math/integration.hpp:29-38) for the
// smooth, piecewise-smooth set-up integrands used here.
double integrate(const std::function<double(double)>& f, double a, double b, double abs_tol, double rel_tol) {
  static const GaussRule lo = gauss_legendre(10);
  static const GaussRule hi = gauss_legendre(21);
  if (a == b) return 0.0;
  struct Seg {
    double a, b, val, err;
  };
  std::vector<Seg> segs;
  auto eval = [&](double x0, double x1) {
    double v1 = rule(hi, f, x0, x1);
    double v0 = rule(lo, f, x0, x1);
    return Seg{x0, x1, v1, std::abs(v1 - v0)};
  };
  segs.push_back(eval(a, b));
  for (int iter = 0; iter < 4000; ++iter) {
    double tot = 0.0, err = 0.0;
    size_t worst = 0;
    for (size_t i = 0; i < segs.size(); ++i) {
      tot += segs[i].val;
      err += segs[i].err;
      if (segs[i].err > segs[worst].err) worst = i;
    }
    if (err <= std::max(abs_tol, rel_tol * std::abs(tot))) return tot;
    Seg s = segs[worst];
    double m = 0.5 * (s.a + s.b);
    segs[worst] = eval(s.a, m);
    segs.push_back(eval(m, s.b));
  }
  double tot = 0.0;
  for (auto& s : segs) tot += s.val;
  return tot;
}

// potentials.hpp:28-37
double hard_sphere_diameter(const Potential& p, double kT, int split) {
  double d_core = hard_core(p);
  double r_split = split_point(p, split);
  auto kernel = [&](double r) { return 1.0 - std::exp(-repulsive(p, r, split) / kT); };
  return d_core + integrate(kernel, d_core, r_split, 1e-12, 1e-12);
}

// potentials.hpp:39-50
double vdw_integral(const Potential& p, double kT, int split) {
  if (p.r_cutoff <= 0.0) return 0.0;
  double r_lower = (split == kBarkerHenderson) ? split_point(p, split) : 0.0;
  auto kernel = [&](double r) { return r * r * attractive(p, r, split); };
  // the integrand has a kink at r_min (WCA); split there for accuracy
  double r_k = split_point(p, split);
  double v = 0.0;
  if (r_k > r_lower && r_k < p.r_cutoff)
    v = integrate(kernel, r_lower, r_k, 1e-13, 1e-13) + integrate(kernel, r_k, p.r_cutoff, 1e-13, 1e-13);
  else
    v = integrate(kernel, r_lower, p.r_cutoff, 1e-13, 1e-13);
  return (2.0 * kPiD / kT) * v;
}

// mean_field.hpp:42-134
double cell_weight(const Potential& p, int split, int scheme, double kT, double dx, long sx, long sy, long sz) {
  return phys::cell_weight(p, split, scheme, kT, dx, sx, sy, sz);
}

// mean_field.hpp:146-196 (before the FFT, which the engine does on the GPU)
double interaction_weight(const long shape[3], double dx, const Potential& p, int split, int scheme, double kT,
                          double* out) {
  const long nx = shape[0], ny = shape[1], nz = shape[2];
  const double dv = dx * dx * dx;
  const double inv_n = 1.0 / static_cast<double>(nx * ny * nz);
  double weight_sum = 0.0;
  for (long ix = 0; ix < nx; ++ix) {
    const long sx = phys::signed_offset(ix, nx);
    for (long iy = 0; iy < ny; ++iy) {
      const long sy = phys::signed_offset(iy, ny);
      for (long iz = 0; iz < nz; ++iz) {
        const long sz = phys::signed_offset(iz, nz);
        const long idx = iz + nz * (iy + ny * ix);
        if (phys::cell_skipped(p, dx, sx, sy, sz)) {
          out[idx] = 0.0;
          continue;
        }
        double w = cell_weight(p, split, scheme, kT, dx, sx, sy, sz);
        out[idx] = w * dv * inv_n;
        weight_sum += w * dv;
      }
    }
  }
  return weight_sum;
}

}  // namespace cdft
