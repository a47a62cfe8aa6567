// Host-side set-up physics (potentials, split schemes, cell weights).
#pragma once

#include <functional>

namespace cdft {

enum PotentialType : int { kLennardJones = 0, kTenWoldeFrenkel = 1, kWRDF = 2 };
enum SplitScheme : int { kWeeksChandlerAndersen = 0, kBarkerHenderson = 1 };
enum WeightScheme : int {
  kWeightZero = 0,
  kWeightLinearE = 1,
  kWeightLinearF = 2,
  kWeightQuadraticF = 3,
  kWeightGaussE = 4,
  kWeightGaussF = 5
};

struct Potential {
  int type = kLennardJones;
  double sigma = 1.0, epsilon = 1.0, r_cutoff = -1.0, alpha = 50.0;
  double epsilon_shift = 0.0;  // for WRDF: the effective epsilon
  double r_min = 0.0, v_min = 0.0, r_zero = 0.0;
};

Potential make_potential(int type, double sigma, double epsilon, double r_cutoff, double alpha);
double raw_potential(const Potential& p, double r);
double split_point(const Potential& p, int split);
double repulsive(const Potential& p, double r, int split);
double attractive(const Potential& p, double r, int split);
double integrate(const std::function<double(double)>& f, double a, double b, double abs_tol, double rel_tol);
double hard_sphere_diameter(const Potential& p, double kT, int split);
double vdw_integral(const Potential& p, double kT, int split);
double cell_weight(const Potential& p, int split, int scheme, double kT, double dx, long sx, long sy, long sz);
// Fills out[N] with the real-space weight * dV / N; returns a_vdw = sum(w dV).
double interaction_weight(const long shape[3], double dx, const Potential& p, int split, int scheme, double kT,
                          double* out);

}  // namespace cdft
