// Bulk (uniform-fluid) thermodynamics of the functional and the phase search
// built on it: include/dft/functionals/bulk/thermodynamics.hpp:14-273 and
// bulk/coexistence.hpp:13-195.  Host code: a few hundred scalar evaluations
// per state point, done once to set up a sweep or a nucleation run.  The
// hard-sphere part evaluates the same templated Phi / dPhi (fmt_models.cuh)
// that the pointwise kernels run on the GPU, at the summed uniform measures.
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>

#include "../../include/cdft_b200.h"
#include "cdft_common.cuh"
#include "fmt_models.cuh"

namespace cdft {
void set_last_error(const std::string& msg);
}  // namespace cdft

namespace {

using cdft::kPi;

void check_model(const cdft_bulk_model* m) {
  if (!m) throw std::invalid_argument("bulk model is NULL");
  if (m->n_species < 1 || m->n_species > CDFT_MAX_SPECIES) throw std::invalid_argument("n_species must be in [1, 4]");
  for (int s = 0; s < m->n_species; ++s)
    if (!(m->diameters[s] > 0.0)) throw std::invalid_argument("hard-sphere diameters must be positive");
  if (m->fmt_model < CDFT_ROSENFELD || m->fmt_model > CDFT_ESFMT) throw std::invalid_argument("unknown FMT model id");
  if (m->n_interactions < 0 || m->n_interactions > CDFT_MAX_INTERACTIONS)
    throw std::invalid_argument("n_interactions must be in [0, 8]");
  for (int k = 0; k < m->n_interactions; ++k) {
    const auto& it = m->interactions[k];
    if (it.species_i < 0 || it.species_i >= m->n_species || it.species_j < 0 || it.species_j >= m->n_species)
      throw std::invalid_argument("interaction species index out of range");
  }
}

// Summed uniform measures of all species (measures.hpp:49-65,
// thermodynamics.hpp:40-50): T = (n2 / 3) I.
cdft::Measures<double> uniform_measures(const cdft_bulk_model& m, const double* rho) {
  cdft::Measures<double> u{};
  for (int s = 0; s < m.n_species; ++s) {
    const double d = m.diameters[s];
    u.eta += (kPi / 6.0) * rho[s] * d * d * d;
    u.n2 += kPi * rho[s] * d * d;
    u.n1 += 0.5 * d * rho[s];
    u.n0 += rho[s];
  }
  const double t = u.n2 / 3.0;
  u.t[0] = u.t[3] = u.t[5] = t;
  return u;
}

// Phi and dPhi of the model at the uniform measures (0 below eta = 1e-30).
bool hs_phi(const cdft_bulk_model& m, const double* rho, double& phi, cdft::MeasureDerivs<double>& dm) {
  const cdft::Measures<double> u = uniform_measures(m, rho);
  phi = 0.0;
  dm = cdft::MeasureDerivs<double>{};
  switch (m.fmt_model) {
    case CDFT_ROSENFELD: return cdft::fmt_phi_dphi<cdft::kRosenfeld, double>(m.esfmt_A, m.esfmt_B, u, phi, dm);
    case CDFT_RSLT: return cdft::fmt_phi_dphi<cdft::kRSLT, double>(m.esfmt_A, m.esfmt_B, u, phi, dm);
    case CDFT_WHITEBEAR_I: return cdft::fmt_phi_dphi<cdft::kWhiteBearI, double>(m.esfmt_A, m.esfmt_B, u, phi, dm);
    case CDFT_WHITEBEAR_II: return cdft::fmt_phi_dphi<cdft::kWhiteBearII, double>(m.esfmt_A, m.esfmt_B, u, phi, dm);
    default: return cdft::fmt_phi_dphi<cdft::kEsFMT, double>(m.esfmt_A, m.esfmt_B, u, phi, dm);
  }
}

// thermodynamics.hpp:201-218
double free_energy_density(const cdft_bulk_model& m, const double* rho) {
  double f = 0.0;
  for (int s = 0; s < m.n_species; ++s)
    if (rho[s] > 0.0) f += rho[s] * (std::log(rho[s]) - 1.0);
  double phi;
  cdft::MeasureDerivs<double> dm;
  if (hs_phi(m, rho, phi, dm)) f += phi;
  double f_mf = 0.0;
  for (int k = 0; k < m.n_interactions; ++k) {
    const auto& it = m.interactions[k];
    f_mf += (it.species_i == it.species_j ? 0.5 : 1.0) * it.a_vdw * rho[it.species_i] * rho[it.species_j];
  }
  return f + f_mf;
}

// thermodynamics.hpp:220-236 (hard-sphere part: thermodynamics.hpp:55-92)
double chemical_potential(const cdft_bulk_model& m, const double* rho, int s) {
  double mu = std::log(rho[s]);
  double phi;
  cdft::MeasureDerivs<double> dm;
  if (hs_phi(m, rho, phi, dm)) {
    const double d = m.diameters[s];
    mu += dm.d_eta * (kPi / 6.0) * d * d * d + dm.d_n2 * kPi * d * d + dm.d_n1 * 0.5 * d + dm.d_n0;
    if (cdft::model_has_tensor(m.fmt_model)) mu += (dm.d_t[0] + dm.d_t[3] + dm.d_t[5]) * (kPi * d * d / 3.0);
  }
  for (int k = 0; k < m.n_interactions; ++k) {
    const auto& it = m.interactions[k];
    if (it.species_i == s && it.species_j == s)
      mu += it.a_vdw * rho[it.species_j];
    else if (it.species_i == s)
      mu += 0.5 * it.a_vdw * rho[it.species_j];
    else if (it.species_j == s)
      mu += 0.5 * it.a_vdw * rho[it.species_i];
  }
  return mu;
}

// thermodynamics.hpp:246-253: P = sum rho_s mu_s - f
double pressure(const cdft_bulk_model& m, const double* rho) {
  double p = -free_energy_density(m, rho);
  for (int s = 0; s < m.n_species; ++s) p += rho[s] * chemical_potential(m, rho, s);
  return p;
}

double pressure1(const cdft_bulk_model& m, double rho) { return pressure(m, &rho); }
double mu1(const cdft_bulk_model& m, double rho) { return chemical_potential(m, &rho, 0); }

// Newton-Raphson in one unknown with the central-difference Jacobian of
// solvers/jacobian.hpp:17-40 (newton.hpp:38-70); false if it does not
// converge or the Jacobian is singular.
template <class F>
bool newton1(double& x, F&& f, int max_iterations, double tolerance) {
  const double eps = 1e-7;
  for (int k = 0; k < max_iterations; ++k) {
    const double fk = f(x);
    if (std::fabs(fk) < tolerance) return true;
    const double J = (f(x + eps) - f(x - eps)) / (2.0 * eps);
    if (!(J != 0.0) || !std::isfinite(J)) return false;
    x -= fk / J;
  }
  return std::fabs(f(x)) < tolerance;
}

// coexistence.hpp:35-49: rho with mu(rho) = target (one species).
bool density_from_mu(const cdft_bulk_model& m, double target, double guess, int max_it, double tol, double& rho) {
  double x = guess;
  const bool ok = newton1(x, [&](double r) { return mu1(m, r) - target; }, max_it, tol);
  if (!ok || !(x > 0.0)) return false;
  rho = x;
  return true;
}

// coexistence.hpp:53-73
double dp_drho(const cdft_bulk_model& m, double rho) {
  const double h = 1e-7;
  return (pressure1(m, rho + h) - pressure1(m, rho - h)) / (2.0 * h);
}

double bisect_dp_drho(const cdft_bulk_model& m, double lo, double hi) {
  double f_lo = dp_drho(m, lo);
  for (int i = 0; i < 60; ++i) {
    const double mid = 0.5 * (lo + hi);
    const double f_mid = dp_drho(m, mid);
    if ((f_lo > 0.0) == (f_mid > 0.0)) {
      lo = mid;
      f_lo = f_mid;
    } else {
      hi = mid;
    }
  }
  return 0.5 * (lo + hi);
}

// coexistence.hpp:77-113: scan dP/drho for its two sign changes, then bisect.
bool find_spinodal(const cdft_bulk_model& m, double rho_max, double step, double& lo_out, double& hi_out) {
  double prev_dp = dp_drho(m, step);
  double low_lo = 0.0, low_hi = 0.0, high_lo = 0.0, high_hi = 0.0;
  bool found_low = false, found_high = false;
  double prev_rho = step;
  for (double rho = 2.0 * step; rho < rho_max; rho += step) {
    const double curr = dp_drho(m, rho);
    if (prev_dp > 0.0 && curr <= 0.0 && !found_low) {
      low_lo = prev_rho;
      low_hi = rho;
      found_low = true;
    } else if (prev_dp < 0.0 && curr >= 0.0 && found_low) {
      high_lo = prev_rho;
      high_hi = rho;
      found_high = true;
      break;
    }
    prev_dp = curr;
    prev_rho = rho;
  }
  if (!found_low || !found_high) return false;
  lo_out = bisect_dp_drho(m, low_lo, low_hi);
  hi_out = bisect_dp_drho(m, high_lo, high_hi);
  return true;
}

// coexistence.hpp:115-191: walk the vapour density down from the low
// spinodal until P_v - P_l(mu_v) changes sign, then bisect it.
bool find_coexistence(const cdft_bulk_model& m, double rho_max, double step, int max_it, double tol, double& rv_out,
                      double& rl_out) {
  double rs1, rs2;
  if (!find_spinodal(m, rho_max, step, rs1, rs2)) return false;
  auto delta_p = [&](double rv, double& dp) {
    double rl;
    if (!density_from_mu(m, mu1(m, rv), rs2 * 1.2, max_it, tol, rl) || rl <= rs2) return false;
    dp = pressure1(m, rv) - pressure1(m, rl);
    return true;
  };
  double rho_v = rs1, dp_prev;
  if (!delta_p(rho_v, dp_prev)) return false;
  double lo = rho_v, hi = rho_v;
  bool bracketed = false;
  while (rho_v > 1e-12) {
    rho_v /= 1.1;
    double dp;
    if (!delta_p(rho_v, dp)) continue;
    if ((dp < 0.0) != (dp_prev < 0.0)) {
      lo = rho_v;
      hi = rho_v * 1.1;
      bracketed = true;
      break;
    }
    dp_prev = dp;
  }
  if (!bracketed) return false;
  double dp_lo;
  if (!delta_p(lo, dp_lo)) return false;
  for (int i = 0; i < 60; ++i) {
    const double mid = 0.5 * (lo + hi);
    double dp_mid;
    if (!delta_p(mid, dp_mid)) {
      hi = mid;
      continue;
    }
    if ((dp_lo > 0.0) == (dp_mid > 0.0)) {
      lo = mid;
      dp_lo = dp_mid;
    } else {
      hi = mid;
    }
  }
  const double rv = 0.5 * (lo + hi);
  double rl;
  if (!density_from_mu(m, mu1(m, rv), rs2 * 1.2, max_it, tol, rl)) return false;
  rv_out = rv;
  rl_out = rl;
  return true;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return CDFT_OK;
  } catch (const std::invalid_argument& e) {
    cdft::set_last_error(e.what());
    return CDFT_ERR_INVALID;
  } catch (const std::exception& e) {
    cdft::set_last_error(e.what());
    return CDFT_ERR_RUNTIME;
  }
}

}  // namespace

extern "C" {

int cdft_bulk_free_energy_density(const cdft_bulk_model* model, const double* rho, double* f) {
  return guarded([&] {
    check_model(model);
    if (!rho || !f) throw std::invalid_argument("rho and f are required");
    *f = free_energy_density(*model, rho);
  });
}

int cdft_bulk_chemical_potentials(const cdft_bulk_model* model, const double* rho, double* mu) {
  return guarded([&] {
    check_model(model);
    if (!rho || !mu) throw std::invalid_argument("rho and mu are required");
    for (int s = 0; s < model->n_species; ++s) mu[s] = chemical_potential(*model, rho, s);
  });
}

int cdft_bulk_pressure(const cdft_bulk_model* model, const double* rho, double* p) {
  return guarded([&] {
    check_model(model);
    if (!rho || !p) throw std::invalid_argument("rho and p are required");
    *p = pressure(*model, rho);
  });
}

int cdft_bulk_density_from_mu(const cdft_bulk_model* model, int n, const double* mu, const double* guess,
                              int max_iterations, double tolerance, double* rho, int* found) {
  return guarded([&] {
    check_model(model);
    if (n < 0 || (n > 0 && (!mu || !guess || !rho || !found))) throw std::invalid_argument("bad arrays");
    for (int i = 0; i < n; ++i) {
      double r = std::numeric_limits<double>::quiet_NaN();
      found[i] = density_from_mu(*model, mu[i], guess[i], max_iterations, tolerance, r) ? 1 : 0;
      rho[i] = r;
    }
  });
}

int cdft_bulk_spinodal(const cdft_bulk_model* model, double rho_max, double rho_scan_step, double out[2],
                       int* found) {
  return guarded([&] {
    check_model(model);
    if (!out || !found) throw std::invalid_argument("out and found are required");
    if (!(rho_scan_step > 0.0) || !(rho_max > 2.0 * rho_scan_step)) throw std::invalid_argument("bad scan range");
    *found = find_spinodal(*model, rho_max, rho_scan_step, out[0], out[1]) ? 1 : 0;
  });
}

int cdft_bulk_coexistence(const cdft_bulk_model* model, double rho_max, double rho_scan_step, int max_iterations,
                          double tolerance, double out[2], int* found) {
  return guarded([&] {
    check_model(model);
    if (!out || !found) throw std::invalid_argument("out and found are required");
    if (!(rho_scan_step > 0.0) || !(rho_max > 2.0 * rho_scan_step)) throw std::invalid_argument("bad scan range");
    *found = find_coexistence(*model, rho_max, rho_scan_step, max_iterations, tolerance, out[0], out[1]) ? 1 : 0;
  });
}

}  // extern "C"
