// C-ABI shim over the reference's own legacy translation
// (legacy/classicaldft.hpp of the reference tree, included from there at
// compile time, never copied): its FMT f-functions, Phi3 and derivatives,
// the full esFMT Phi, the QF mean-field weights and a_vdw, the Enskog
// hard-sphere thermodynamics and the spinodal / coexistence solver.  Built
// by oracle/build_ref.py into oracle/_ref/liblegacy_ref.so; the oracle's
// tests call it through ctypes to pin the oracle's restatement against code
// of the reference itself.  Test infrastructure only.
#include <stdexcept>

#include "legacy/classicaldft.hpp"

namespace {

namespace lf = legacy::fmt;

// model ids: 0 Rosenfeld, 1 RSLT, 2 esFMT, 3 WhiteBearI, 4 WhiteBearII
double f_of(int model, int which, double x) {
  switch (model) {
    case 0: return which == 1 ? lf::Rosenfeld_model::f1(x) : which == 2 ? lf::Rosenfeld_model::f2(x)
                                                                         : lf::Rosenfeld_model::f3(x);
    case 1: return which == 1 ? lf::RSLT_model::f1(x) : which == 2 ? lf::RSLT_model::f2(x) : lf::RSLT_model::f3(x);
    case 2: return which == 1 ? lf::esFMT_model::f1(x) : which == 2 ? lf::esFMT_model::f2(x)
                                                                     : lf::esFMT_model::f3(x);
    case 3: return which == 1 ? lf::WhiteBearI_model::f1(x) : which == 2 ? lf::WhiteBearI_model::f2(x)
                                                                           : lf::WhiteBearI_model::f3(x);
    case 4: return which == 1 ? lf::WhiteBearII_model::f1(x) : which == 2 ? lf::WhiteBearII_model::f2(x)
                                                                            : lf::WhiteBearII_model::f3(x);
    default: throw std::invalid_argument("model");
  }
}

// in: eta, s0, s1, s2, v1[3], v2[3], T[3][3] (row-major): 19 doubles
lf::FundamentalMeasures measures(const double* in) {
  lf::FundamentalMeasures fm;
  fm.eta = in[0];
  fm.s0 = in[1];
  fm.s1 = in[2];
  fm.s2 = in[3];
  for (int i = 0; i < 3; ++i) {
    fm.v1[i] = in[4 + i];
    fm.v2[i] = in[7 + i];
    for (int j = 0; j < 3; ++j) fm.T[i][j] = in[10 + 3 * i + j];
  }
  fm.calculate_derived_quantities();
  return fm;
}

}  // namespace

extern "C" {

double lref_f(int model, int which, double x) { return f_of(model, which, x); }

double lref_fex(int model, double eta, double A, double B) {
  switch (model) {
    case 0: return lf::Rosenfeld_model::fex(eta);
    case 1: return lf::RSLT_model::fex(eta);
    case 2: return lf::esFMT_model::fex(eta, A, B);
    case 3: return lf::WhiteBearI_model::fex(eta);
    case 4: return lf::WhiteBearII_model::fex(eta);
    default: return 0.0;
  }
}

// derived: v1_v2, v2_v2, vTv, T2, T3, vT[3], Tv[3], TT[3][3] (20 doubles)
void lref_derived(const double* in, double* out) {
  const lf::FundamentalMeasures fm = measures(in);
  out[0] = fm.v1_v2;
  out[1] = fm.v2_v2;
  out[2] = fm.vTv;
  out[3] = fm.T2;
  out[4] = fm.T3;
  for (int i = 0; i < 3; ++i) {
    out[5 + i] = fm.vT[i];
    out[8 + i] = fm.Tv[i];
    for (int j = 0; j < 3; ++j) out[11 + 3 * i + j] = fm.TT[i][j];
  }
}

// Phi3 and its derivatives of model 0 (Rosenfeld), 1 (RSLT) or 2 (esFMT, A, B):
// out = {Phi3, dPhi3/ds2, dPhi3/dv2[0..2], dPhi3/dT[j][k] (esFMT only, 9)}
void lref_phi3(int model, double A, double B, const double* in, double* out) {
  const lf::FundamentalMeasures fm = measures(in);
  for (int t = 0; t < 14; ++t) out[t] = 0.0;
  if (model == 0) {
    out[0] = lf::Rosenfeld_model::Phi3(fm);
    out[1] = lf::Rosenfeld_model::dPhi3_dS2(fm);
    for (int k = 0; k < 3; ++k) out[2 + k] = lf::Rosenfeld_model::dPhi3_dV2(k, fm);
  } else if (model == 1) {
    out[0] = lf::RSLT_model::Phi3(fm);
    out[1] = lf::RSLT_model::dPhi3_dS2(fm);
    for (int k = 0; k < 3; ++k) out[2 + k] = lf::RSLT_model::dPhi3_dV2(k, fm);
  } else {
    out[0] = lf::esFMT_model::Phi3(A, B, fm);
    out[1] = lf::esFMT_model::dPhi3_dS2(A, B, fm);
    for (int k = 0; k < 3; ++k) out[2 + k] = lf::esFMT_model::dPhi3_dV2(A, k, fm);
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) out[5 + 3 * j + k] = lf::esFMT_model::dPhi3_dT(A, B, j, k, fm);
  }
}

double lref_phi(const double* in, double A, double B) { return lf::phi(measures(in), A, B); }

double lref_watt2_lj(double sigma, double eps, double rcut, double r2) {
  return legacy::interactions::Watt2_LJ(sigma, eps, rcut, r2);
}

double lref_weight_qf(double sigma, double eps, double rcut, int sx, int sy, int sz, double dx) {
  return legacy::interactions::generate_weight_QF(sigma, eps, rcut, sx, sy, sz, dx);
}

double lref_avdw_qf(double sigma, double eps, double rcut, double kT, double dx) {
  return legacy::interactions::compute_a_vdw_QF(sigma, eps, rcut, kT, dx);
}

// Enskog (Percus-Yevick compressibility / Carnahan-Starling) at density n:
// {exFreeEnergyPYC, exFreeEnergyCS, pressurePYC, pressureCS, freeEnergyPYC,
//  chemPotentialPYC, dexFreeEnergyPYCdRho, dexFreeEnergyCSdRho}
void lref_enskog(double n, double* out) {
  const legacy::thermodynamics::Enskog e(n);
  out[0] = e.exFreeEnergyPYC();
  out[1] = e.exFreeEnergyCS();
  out[2] = e.pressurePYC();
  out[3] = e.pressureCS();
  out[4] = e.freeEnergyPYC();
  out[5] = e.chemPotentialPYC();
  out[6] = e.dexFreeEnergyPYCdRho();
  out[7] = e.dexFreeEnergyCSdRho();
}

typedef double (*lref_scalar_fn)(double x, void* user);

// findSpinodal / findCoex on the caller's pressure and chemical potential;
// returns 0, or 1 when the solver threw (out untouched).
int lref_spinodal(lref_scalar_fn pressure, lref_scalar_fn chem, void* user, double xmax, double dx, double tol,
                  double* out) {
  legacy::solver::EOS eos{[=](double x) { return pressure(x, user); }, [=](double x) { return chem(x, user); }};
  try {
    const auto s = legacy::solver::findSpinodal(eos, xmax, dx, tol);
    out[0] = s.xs1;
    out[1] = s.xs2;
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

int lref_coexistence(lref_scalar_fn pressure, lref_scalar_fn chem, void* user, double xmax, double dx, double tol,
                     double* out) {
  legacy::solver::EOS eos{[=](double x) { return pressure(x, user); }, [=](double x) { return chem(x, user); }};
  try {
    const auto c = legacy::solver::findCoex(eos, xmax, dx, tol);
    out[0] = c.x1;
    out[1] = c.x2;
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

}  // extern "C"
