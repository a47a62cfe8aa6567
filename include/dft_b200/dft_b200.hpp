// C++ host API of the classicalDFT B200 engine: the reference's functional,
// grid, minimiser, Picard, DDFT, saddle-point and lattice interfaces
// (namespaces and names of include/dft/{grid,types}.hpp,
// functionals/{functionals,functional}.hpp,
// algorithms/{fire,minimization,picard,dynamics,saddle_point}.hpp,
// src/crystal.cpp) over the C ABI of cdft_b200.h.  Fields are std::vector<double> in the reference's layout
// (z fastest); device copies are made per call.  Errors are thrown as the
// reference's exception types: std::invalid_argument / std::runtime_error.
//
// Header-only; link with -lcdft_b200 -lcudart.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../cdft_b200.h"

namespace dft_b200 {

inline void check(int status) {
  if (status == CDFT_OK) return;
  const std::string msg = cdft_last_error();
  if (status == CDFT_ERR_INVALID) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

inline void cuda_check(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
}

// A device copy of a host vector, freed on scope exit.
class DeviceVector {
 public:
  explicit DeviceVector(std::size_t n) : n_(n) { cuda_check(cudaMalloc(&p_, sizeof(double) * (n ? n : 1))); }
  explicit DeviceVector(const std::vector<double>& h) : DeviceVector(h.size()) { upload(h); }
  ~DeviceVector() { cudaFree(p_); }
  DeviceVector(const DeviceVector&) = delete;
  DeviceVector& operator=(const DeviceVector&) = delete;
  void upload(const std::vector<double>& h) {
    cuda_check(cudaMemcpy(p_, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
  }
  std::vector<double> download() const {
    std::vector<double> h(n_);
    cuda_check(cudaMemcpy(h.data(), p_, sizeof(double) * n_, cudaMemcpyDeviceToHost));
    return h;
  }
  double* get() const { return p_; }

 private:
  double* p_ = nullptr;
  std::size_t n_ = 0;
};

// ---------------------------------------------------------------- grid.hpp

struct Grid {
  double dx = 0.0;
  std::array<double, 3> box_size{};
  std::array<long, 3> shape{};
  double cell_volume() const { return dx * dx * dx; }
  long total_points() const { return shape[0] * shape[1] * shape[2]; }
  long flat_index(long ix, long iy, long iz) const { return iz + shape[2] * (iy + shape[1] * ix); }
  std::vector<unsigned char> boundary_mask() const {
    std::vector<unsigned char> m(static_cast<std::size_t>(total_points()), 0);
    for (long ix = 0; ix < shape[0]; ++ix)
      for (long iy = 0; iy < shape[1]; ++iy)
        for (long iz = 0; iz < shape[2]; ++iz)
          if (ix == 0 || ix == shape[0] - 1 || iy == 0 || iy == shape[1] - 1 || iz == 0 || iz == shape[2] - 1)
            m[static_cast<std::size_t>(flat_index(ix, iy, iz))] = 1;
    return m;
  }
};

// grid.hpp:87-108
inline Grid make_grid(double dx, std::array<double, 3> box) {
  if (dx <= 0.0) throw std::invalid_argument("make_grid: dx must be positive, got " + std::to_string(dx));
  Grid g{dx, box, {}};
  for (int d = 0; d < 3; ++d) {
    if (box[d] <= 0.0) throw std::invalid_argument("make_grid: box dimension must be positive");
    const double n = box[d] / dx;
    const long ni = static_cast<long>(std::round(n));
    if (std::abs(n - static_cast<double>(ni)) > 1e-10)
      throw std::invalid_argument("make_grid: box dimension " + std::to_string(box[d]) +
                                  " is not commensurate with dx=" + std::to_string(dx));
    g.shape[d] = ni;
  }
  return g;
}

// ------------------------------------------------------------- physics

namespace physics {

enum class SplitScheme { WeeksChandlerAndersen = CDFT_SPLIT_WCA, BarkerHenderson = CDFT_SPLIT_BH };
enum class WeightScheme {
  InterpolationZero = CDFT_WEIGHT_ZERO,
  InterpolationLinearE = CDFT_WEIGHT_LINEAR_E,
  InterpolationLinearF = CDFT_WEIGHT_LINEAR_F,
  InterpolationQuadraticF = CDFT_WEIGHT_QUADRATIC_F,
  GaussE = CDFT_WEIGHT_GAUSS_E,
  GaussF = CDFT_WEIGHT_GAUSS_F,
};

// potentials.hpp:248-307 (the variant's parameters)
struct Potential {
  cdft_potential p{CDFT_POT_LENNARD_JONES, 1.0, 1.0, -1.0, 50.0};
  double attractive(double r, SplitScheme s = SplitScheme::WeeksChandlerAndersen) const {
    double out = 0.0;
    check(cdft_potential_attractive(&p, static_cast<int>(s), &r, 1, &out));
    return out;
  }
  double hard_sphere_diameter(double kT, SplitScheme s = SplitScheme::WeeksChandlerAndersen) const {
    double d = 0.0;
    check(cdft_hard_sphere_diameter(&p, kT, static_cast<int>(s), &d));
    return d;
  }
  double vdw_integral(double kT, SplitScheme s = SplitScheme::WeeksChandlerAndersen) const {
    double v = 0.0;
    check(cdft_vdw_integral(&p, kT, static_cast<int>(s), &v));
    return v;
  }
};

inline Potential make_lennard_jones(double sigma, double epsilon, double r_cutoff = -1.0) {
  return Potential{{CDFT_POT_LENNARD_JONES, sigma, epsilon, r_cutoff, 50.0}};
}
inline Potential make_ten_wolde_frenkel(double sigma, double epsilon, double r_cutoff = -1.0, double alpha = 50.0) {
  return Potential{{CDFT_POT_TEN_WOLDE_FRENKEL, sigma, epsilon, r_cutoff, alpha}};
}
inline Potential make_wang_ramirez_dobnikar_frenkel(double sigma, double epsilon, double r_cutoff = 3.0) {
  return Potential{{CDFT_POT_WRDF, sigma, epsilon, r_cutoff, 50.0}};
}

// interactions.hpp:23-30
struct Interaction {
  int species_i = 0, species_j = 0;
  Potential potential;
  SplitScheme split = SplitScheme::WeeksChandlerAndersen;
  WeightScheme weight_scheme = WeightScheme::InterpolationQuadraticF;
};

struct Species {
  std::string name;
  double hard_sphere_diameter = 1.0;
};

// model.hpp:15-20
struct Model {
  Grid grid;
  std::vector<Species> species;
  std::vector<Interaction> interactions;
  double temperature = 1.0;
};

}  // namespace physics

// ---------------------------------------------------------- functionals

namespace functionals {

// models.hpp:363-419 (as a tag plus esFMT's A, B)
struct FMTModel {
  int id = CDFT_WHITEBEAR_II;
  double A = 1.0, B = 0.0;
  static FMTModel Rosenfeld() { return {CDFT_ROSENFELD}; }
  static FMTModel RSLT() { return {CDFT_RSLT}; }
  static FMTModel WhiteBearI() { return {CDFT_WHITEBEAR_I}; }
  static FMTModel WhiteBearII() { return {CDFT_WHITEBEAR_II}; }
  static FMTModel EsFMT(double a = 1.0, double b = 0.0) { return {CDFT_ESFMT, a, b}; }
};

// functionals.hpp:19-23: the GPU-resident weights of one (FMT model, Model).
class Weights {
 public:
  Weights(const FMTModel& fmt, const physics::Model& model, int precision = CDFT_FP64) : fmt_(fmt) {
    const auto& g = model.grid;
    std::vector<double> d;
    for (const auto& sp : model.species) d.push_back(sp.hard_sphere_diameter);
    std::vector<cdft_model_interaction> inter;
    for (const auto& it : model.interactions)  // mean_field.hpp:146-196, made on the GPU
      inter.push_back({it.species_i, it.species_j, it.potential.p, static_cast<int>(it.split),
                       static_cast<int>(it.weight_scheme)});
    cdft_engine* e = nullptr;
    check(cdft_create_model(&e, g.shape.data(), g.dx, static_cast<int>(d.size()), d.data(), fmt.id, fmt.A, fmt.B,
                            static_cast<int>(inter.size()), inter.empty() ? nullptr : inter.data(),
                            model.temperature, precision, 1));
    engine_.reset(e);
    for (int m = 0; m < static_cast<int>(inter.size()); ++m) {
      double a = 0.0;
      check(cdft_engine_a_vdw(e, m, &a));
      a_vdw_.push_back(a);
    }
  }
  cdft_engine* engine() const { return engine_.get(); }
  const std::vector<double>& a_vdw() const { return a_vdw_; }
  // Anchored split of a mixed-precision Weights (cdft_engine_set_anchor_host):
  // later evaluations transform rho - rho_anchor in FP32 around the FP64
  // fields of rho_anchor, evaluated once by `fp64` (an FP64 Weights of the
  // same model).  rho_anchor: S*N values, species after species.
  void set_anchor(const Weights& fp64, const std::vector<double>& rho_anchor) {
    check(cdft_engine_set_anchor_host(engine(), fp64.engine(), rho_anchor.data()));
  }
  void clear_anchor() { check(cdft_engine_clear_anchor(engine())); }
  const FMTModel& fmt_model() const { return fmt_; }

 private:
  struct Del {
    void operator()(cdft_engine* e) const { cdft_destroy(e); }
  };
  FMTModel fmt_;
  std::unique_ptr<cdft_engine, Del> engine_;
  std::vector<double> a_vdw_;
};

inline Weights make_weights(const FMTModel& fmt, const physics::Model& model, int precision = CDFT_FP64) {
  return Weights(fmt, model, precision);
}

// types.hpp:17-48 (one species' state)
struct SpeciesState {
  std::vector<double> values;          // density
  std::vector<double> external_field;  // empty: no field
  double chemical_potential = 0.0;     // beta mu
};
struct State {
  std::vector<SpeciesState> species;
  double temperature = 1.0;
};

// functionals/types.hpp:18-23
struct Result {
  double free_energy = 0.0;
  double grand_potential = 0.0;
  std::vector<std::vector<double>> forces;
};

// functionals.hpp:64-95
inline Result total(const physics::Model& model, const State& state, const Weights& weights) {
  const std::size_t S = state.species.size();
  const std::size_t N = static_cast<std::size_t>(model.grid.total_points());
  if (S != model.species.size()) throw std::invalid_argument("total: one SpeciesState per species");
  std::vector<double> rho(S * N), vext, mu(S), force(S * N), sc(CDFT_SCALAR_COUNT);
  bool field = false;
  for (const auto& sp : state.species) field = field || !sp.external_field.empty();
  if (field) vext.assign(S * N, 0.0);
  for (std::size_t s = 0; s < S; ++s) {
    const auto& sp = state.species[s];
    if (sp.values.size() != N) throw std::invalid_argument("total: density has the wrong size");
    std::memcpy(rho.data() + s * N, sp.values.data(), sizeof(double) * N);
    if (!sp.external_field.empty()) {
      if (sp.external_field.size() != N) throw std::invalid_argument("total: external field has the wrong size");
      std::memcpy(vext.data() + s * N, sp.external_field.data(), sizeof(double) * N);
    }
    mu[s] = sp.chemical_potential;
  }
  check(cdft_total(weights.engine(), rho.data(), field ? vext.data() : nullptr, mu.data(), force.data(), sc.data()));
  Result r;
  r.free_energy = sc[0];
  r.grand_potential = sc[1];
  for (std::size_t s = 0; s < S; ++s) r.forces.emplace_back(force.begin() + s * N, force.begin() + (s + 1) * N);
  return r;
}

// `total` for a sequence of states (cdft_total_stream): the copies of one
// state overlap the evaluation of the next; one Result per state, equal to
// `total` on each.
inline std::vector<Result> total_stream(const physics::Model& model, const std::vector<State>& states,
                                        const Weights& weights) {
  const std::size_t S = model.species.size();
  const std::size_t N = static_cast<std::size_t>(model.grid.total_points());
  const std::size_t K = states.size();
  std::vector<std::vector<double>> rho(K), vext(K), force(K, std::vector<double>(S * N));
  std::vector<const double*> rp(K), vp(K, nullptr);
  std::vector<double*> fp(K);
  std::vector<double> mu(K * S), sc(K * CDFT_SCALAR_COUNT);
  for (std::size_t i = 0; i < K; ++i) {
    const State& st = states[i];
    if (st.species.size() != S) throw std::invalid_argument("total_stream: one SpeciesState per species");
    rho[i].resize(S * N);
    for (std::size_t s = 0; s < S; ++s) {
      const auto& sp = st.species[s];
      if (sp.values.size() != N) throw std::invalid_argument("total_stream: density has the wrong size");
      std::memcpy(rho[i].data() + s * N, sp.values.data(), sizeof(double) * N);
      if (!sp.external_field.empty()) {
        if (sp.external_field.size() != N)
          throw std::invalid_argument("total_stream: external field has the wrong size");
        if (vext[i].empty()) vext[i].assign(S * N, 0.0);
        std::memcpy(vext[i].data() + s * N, sp.external_field.data(), sizeof(double) * N);
      }
      mu[i * S + s] = sp.chemical_potential;
    }
    rp[i] = rho[i].data();
    vp[i] = vext[i].empty() ? nullptr : vext[i].data();
    fp[i] = force[i].data();
  }
  check(cdft_total_stream(weights.engine(), static_cast<int>(K), rp.data(), vp.data(), mu.data(), fp.data(),
                          sc.data()));
  std::vector<Result> out(K);
  for (std::size_t i = 0; i < K; ++i) {
    out[i].free_energy = sc[i * CDFT_SCALAR_COUNT];
    out[i].grand_potential = sc[i * CDFT_SCALAR_COUNT + 1];
    for (std::size_t s = 0; s < S; ++s)
      out[i].forces.emplace_back(force[i].begin() + s * N, force[i].begin() + (s + 1) * N);
  }
  return out;
}

using ForceCallback = std::function<std::pair<double, std::vector<std::vector<double>>>(
    const std::vector<std::vector<double>>&)>;

// functional.hpp:22-107
struct Functional {
  physics::Model model;
  std::shared_ptr<Weights> weights;

  Functional(const FMTModel& fmt, physics::Model m, int precision = CDFT_FP64)
      : model(std::move(m)), weights(std::make_shared<Weights>(fmt, model, precision)) {}

  Result evaluate(const State& state) const { return total(model, state, *weights); }

  // functional.hpp:33-36: the external field is zero (init::from_profile)
  Result evaluate(const std::vector<double>& rho, double chemical_potential) const {
    State st;
    st.temperature = model.temperature;
    st.species.push_back({rho, {}, chemical_potential});
    for (std::size_t s = 1; s < model.species.size(); ++s)
      st.species.push_back({std::vector<double>(rho.size(), 0.0), {}, 0.0});
    return total(model, st, *weights);
  }

  double grand_potential(const std::vector<double>& rho, double mu) const { return evaluate(rho, mu).grand_potential; }

  // functional.hpp:62-73
  ForceCallback grand_potential_callback(double chemical_potential) const {
    auto self = *this;
    return [self, chemical_potential](const std::vector<std::vector<double>>& dens) {
      State st;
      st.temperature = self.model.temperature;
      for (const auto& d : dens) st.species.push_back({d, {}, chemical_potential});
      auto r = total(self.model, st, *self.weights);
      return std::make_pair(r.grand_potential, r.forces);
    };
  }
};

}  // namespace functionals

// ----------------------------------------------------------- algorithms

namespace algorithms {

namespace fire {
// fire.hpp:33-44
struct Fire {
  double dt = 1e-3, dt_max = 1e-2, dt_min = 1e-8, alpha_start = 0.1, f_inc = 1.1, f_dec = 0.5, f_alpha = 0.99;
  int n_delay = 5, max_uphill = 20;
  double force_tolerance = 0.1;
  int max_steps = 10000;
  cdft_fire_params c() const {
    return {dt, dt_max, dt_min, alpha_start, f_inc, f_dec, f_alpha, n_delay, max_uphill, force_tolerance, max_steps};
  }
};
}  // namespace fire

namespace minimization {

struct Unbounded {
  double rho_min = 1e-18;
};
struct Bounded {
  double rho_min = 1e-18, rho_max = 1.0;
};

// minimization.hpp:114-121
struct Result {
  std::vector<std::vector<double>> densities;
  double free_energy = 0.0, grand_potential = 0.0, rms_force = 0.0;
  int iterations = 0;
  bool converged = false;
};

// minimization.hpp:123-147; runs on the device (cdft_minimize)
struct Minimizer {
  fire::Fire fire{};
  bool bounded = false;
  Unbounded unbounded{};
  Bounded bounded_param{};
  bool use_homogeneous_boundary = true;
  int check_interval = 25;
  const functionals::Weights* refine = nullptr;  // optional FP64 defect correction
  double refine_switch = 10.0;
  // true: the energy monitor (minimization.hpp:431-434); false: the rms force (fire.hpp:162)
  bool use_monitor = true;
  // V_ext of every evaluation (N values), or empty; the reference's
  // Minimizer has none (init.hpp:28-58 drops it), a wall needs it
  std::vector<double> external_field;

  Result run(const functionals::Weights& w, const std::vector<double>& rho0, int mode, double mu, double mass) const {
    cdft_minimizer_config cfg{};
    cfg.fire = fire.c();
    cfg.mode = mode;
    cfg.parametrization = bounded ? CDFT_PARAM_BOUNDED : CDFT_PARAM_UNBOUNDED;
    cfg.rho_min = bounded ? bounded_param.rho_min : unbounded.rho_min;
    cfg.rho_max = bounded ? bounded_param.rho_max : 1.0;
    cfg.homogeneous_boundary = use_homogeneous_boundary ? 1 : 0;
    cfg.chemical_potential = mu;
    cfg.target_mass = mass;
    cfg.use_monitor = use_monitor ? 1 : 0;
    cfg.check_interval = check_interval;
    DeviceVector d(rho0);
    DeviceVector vx(external_field.empty() ? std::vector<double>(1, 0.0) : external_field);
    cfg.external_field = external_field.empty() ? nullptr : vx.get();
    cdft_minimizer_result res{};
    check(cdft_minimize(w.engine(), &cfg, d.get(), nullptr, refine ? refine->engine() : nullptr, refine_switch, &res,
                        nullptr));
    Result r;
    r.densities.push_back(d.download());
    r.free_energy = res.free_energy;
    r.grand_potential = res.grand_potential;
    r.rms_force = res.rms_force;
    r.iterations = res.iterations;
    r.converged = res.converged != 0;
    return r;
  }
  // minimization.hpp:182-278
  Result fixed_mass(const physics::Model&, const functionals::Weights& w, const std::vector<double>& rho0, double mu,
                    double target_mass) const {
    return run(w, rho0, CDFT_MIN_FIXED_MASS, mu, target_mass);
  }
  // minimization.hpp:280-354
  Result grand_potential(const physics::Model&, const functionals::Weights& w, const std::vector<double>& rho0,
                         double mu) const {
    return run(w, rho0, CDFT_MIN_GRAND_POTENTIAL, mu, 0.0);
  }
};

}  // namespace minimization

namespace picard {

// picard.hpp:23-29
struct PicardResult {
  std::vector<std::vector<double>> densities;
  double grand_potential = 0.0, residual = 0.0;
  int iterations = 0;
  bool converged = false;
};

// minimization.hpp:159-180: the excess over the background rescaled to the
// target mass after every update
struct Constraint {
  std::vector<double> target_masses;
  std::vector<std::vector<double>> backgrounds;
  double cell_volume = 0.0, min_density = 1e-30;
};
inline Constraint fixed_mass_constraint(std::vector<double> target_masses,
                                        std::vector<std::vector<double>> backgrounds, double cell_volume,
                                        double min_density = 1e-30) {
  return Constraint{std::move(target_masses), std::move(backgrounds), cell_volume, min_density};
}

// picard.hpp:31-124 on the device (log_interval kept for the interface;
// nothing is printed)
struct Picard {
  double mixing = 0.01, min_density = 1e-30, tolerance = 1e-6;
  int max_iterations = 5000, log_interval = 500;
  int check_interval = 25;

  PicardResult solve(std::vector<std::vector<double>> densities, const functionals::Weights& w,
                     double chemical_potential, const Constraint* constraint = nullptr) const {
    const std::vector<double>& rho = densities.at(0);
    DeviceVector d(rho);
    cdft_picard_config cfg{mixing, min_density, tolerance, constraint ? constraint->min_density : 1e-30,
                           max_iterations, check_interval};
    cdft_picard_result res{};
    std::unique_ptr<DeviceVector> bg;
    double mass = 0.0;
    if (constraint) {
      if (constraint->target_masses.empty()) throw std::invalid_argument("fixed_mass_constraint: no target mass");
      mass = constraint->target_masses[0];
      if (!constraint->backgrounds.empty()) {
        if (constraint->backgrounds[0].size() != rho.size())
          throw std::invalid_argument("fixed_mass_constraint: background has the wrong size");
        bg = std::make_unique<DeviceVector>(constraint->backgrounds[0]);
      }
    }
    check(cdft_picard(w.engine(), &cfg, &chemical_potential, constraint ? &mass : nullptr, bg ? bg->get() : nullptr,
                      d.get(), &res, nullptr));
    PicardResult r;
    r.densities.push_back(d.download());
    r.grand_potential = res.grand_potential;
    r.residual = res.residual;
    r.iterations = res.iterations;
    r.converged = res.converged != 0;
    return r;
  }
};

}  // namespace picard

namespace dynamics {

// dynamics.hpp:26-33
struct StepConfig {
  double dt = 1e-4, diffusion_coefficient = 1.0, min_density = 1e-18, dt_max = 1.0, fp_tolerance = 1e-4;
  int fp_max_iterations = 100;
  cdft_ddft_config c() const { return {dt, diffusion_coefficient, min_density, dt_max, fp_tolerance, fp_max_iterations}; }
};

// dynamics.hpp:36-40
struct StepResult {
  std::vector<std::vector<double>> densities;
  double energy = 0.0;
  double dt_used = 0.0;
};

namespace detail {
template <class F>
StepResult one_step(const std::vector<std::vector<double>>& densities, F&& call) {
  DeviceVector d(densities.at(0));
  StepResult r;
  r.dt_used = call(d.get(), &r.energy);
  r.densities.push_back(d.download());
  return r;
}
}  // namespace detail

// dynamics.hpp:333-401 (config.dt is divided by 10 on every restart)
inline StepResult integrating_factor_step(const std::vector<std::vector<double>>& densities,
                                          const functionals::Weights& w, StepConfig& config,
                                          double chemical_potential = 0.0) {
  return detail::one_step(densities, [&](double* d, double* e) {
    cdft_ddft_config c = config.c();
    check(cdft_ddft_step(w.engine(), &c, chemical_potential, d, e, nullptr, nullptr));
    config.dt = c.dt;
    return c.dt;
  });
}

// dynamics.hpp:410-465
inline StepResult split_operator_step(const std::vector<std::vector<double>>& densities,
                                      const functionals::Weights& w, const StepConfig& config,
                                      double chemical_potential = 0.0) {
  return detail::one_step(densities, [&](double* d, double* e) {
    const cdft_ddft_config c = config.c();
    check(cdft_ddft_split_step(w.engine(), &c, chemical_potential, d, e, nullptr));
    return c.dt;
  });
}

// dynamics.hpp:472-538
inline StepResult crank_nicholson_step(const std::vector<std::vector<double>>& densities,
                                       const functionals::Weights& w, const StepConfig& config,
                                       double chemical_potential = 0.0) {
  return detail::one_step(densities, [&](double* d, double* e) {
    const cdft_ddft_config c = config.c();
    check(cdft_ddft_cn_step(w.engine(), &c, chemical_potential, d, e, nullptr, nullptr));
    return c.dt;
  });
}

// dynamics.hpp:45-50
struct Snapshot {
  int step = 0;
  double time = 0.0, energy = 0.0;
  std::vector<std::vector<double>> densities;
};

// dynamics.hpp:54-61
struct SimulationResult {
  std::vector<std::vector<double>> densities;
  std::vector<double> times, energies;
  std::vector<Snapshot> snapshots;
  double mass_initial = 0.0, mass_final = 0.0;
};

// dynamics.hpp:551-557: the masked cells are reset to the reservoir density
// after every step (an empty mask: periodic, canonical).
struct BoundaryCondition {
  std::vector<unsigned char> mask;
  double reservoir_density = 0.0;
  explicit operator bool() const { return !mask.empty(); }
};
inline BoundaryCondition reservoir_boundary(const std::vector<unsigned char>& mask, double reservoir_density) {
  return BoundaryCondition{mask, reservoir_density};
}

using StopCondition = std::function<bool(int step, double time, double energy)>;

// dynamics.hpp:564-693 (integrating-factor DDFT on the device; snapshots are
// copied to pinned host memory while the following steps run).  times and
// energies hold the entries the reference records (step 0, every
// log_interval-th step and the last); nothing is printed.
struct Simulation {
  StepConfig step;
  int n_steps = 1000;
  int snapshot_interval = 100;
  int log_interval = 50;
  double energy_offset = 0.0;
  BoundaryCondition boundary{};
  StopCondition stop_condition{};

  SimulationResult run(std::vector<std::vector<double>> densities, const Grid& grid, const functionals::Weights& w,
                       double chemical_potential) const {
    const std::size_t N = static_cast<std::size_t>(grid.total_points());
    auto& rho0 = densities.at(0);
    if (rho0.size() != N) throw std::invalid_argument("Simulation::run: density has the wrong size");
    if (boundary) {
      if (boundary.mask.size() != N) throw std::invalid_argument("reservoir mask: one entry per grid point");
      for (std::size_t i = 0; i < N; ++i)
        if (boundary.mask[i]) rho0[i] = boundary.reservoir_density;
    }
    SimulationResult r;
    double m0 = 0.0;
    for (double v : rho0) m0 += v;
    r.mass_initial = m0 * grid.cell_volume();
    DeviceVector d(rho0);
    unsigned char* mask = nullptr;
    if (boundary) {
      cuda_check(cudaMalloc(&mask, N));
      cuda_check(cudaMemcpy(mask, boundary.mask.data(), N, cudaMemcpyHostToDevice));
    }
    const int cap = snapshot_interval > 0 ? 1 + n_steps / snapshot_interval : 0;
    double* snaps = nullptr;
    std::vector<int> snap_steps(static_cast<std::size_t>(cap > 0 ? cap : 1));
    if (cap > 0) {
      const cudaError_t e = cudaMallocHost(&snaps, sizeof(double) * N * static_cast<std::size_t>(cap));
      if (e != cudaSuccess) {
        cudaFree(mask);
        cuda_check(e);
      }
    }
    std::vector<double> times(static_cast<std::size_t>(n_steps) + 1), energies(times.size());
    struct Ctx {
      const StopCondition* f;
      std::exception_ptr err;
    } ctx{&stop_condition, nullptr};
    auto tramp = [](int s, double t, double e, void* user) -> int {
      auto* c = static_cast<Ctx*>(user);
      try {
        return (*c->f)(s, t, e) ? 1 : 0;
      } catch (...) {
        c->err = std::current_exception();
        return 1;
      }
    };
    cdft_ddft_config c = step.c();
    int count = 0, done = 0;
    const int status = cdft_ddft_simulate(w.engine(), &c, chemical_potential, n_steps, d.get(), times.data(),
                                          energies.data(), snapshot_interval, snaps, snap_steps.data(), cap, &count,
                                          mask, boundary.reservoir_density, stop_condition ? +tramp : nullptr,
                                          &ctx, &done, nullptr);
    cudaFree(mask);
    for (int k = 0; k < count; ++k) {
      const int st = snap_steps[static_cast<std::size_t>(k)];
      Snapshot sn{st, times[static_cast<std::size_t>(st)], energies[static_cast<std::size_t>(st)], {}};
      sn.densities.emplace_back(snaps + static_cast<std::size_t>(k) * N, snaps + static_cast<std::size_t>(k + 1) * N);
      r.snapshots.push_back(std::move(sn));
    }
    if (snaps) cudaFreeHost(snaps);
    check(status);
    if (ctx.err) std::rethrow_exception(ctx.err);
    r.times.push_back(times[0]);
    r.energies.push_back(energies[0]);
    for (int s = 1; s <= done; ++s)
      if (log_interval > 0 && (s % log_interval == 0 || s == n_steps)) {
        r.times.push_back(times[static_cast<std::size_t>(s)]);
        r.energies.push_back(energies[static_cast<std::size_t>(s)]);
      }
    r.densities.push_back(d.download());
    double m1 = 0.0;
    for (double v : r.densities[0]) m1 += v;
    r.mass_final = m1 * grid.cell_volume();
    return r;
  }
};

}  // namespace dynamics

namespace saddle_point {

struct EigenvalueResult {
  std::vector<double> eigenvector;
  double eigenvalue = 0.0;
  int iterations = 0;
  bool converged = false;
};

// saddle_point.hpp:158-169 (exact_hvp replaces the finite difference).
// method CDFT_EIGEN_LANCZOS: block Lanczos on exact products of the same
// operator, `block` directions per batched product taken from `hvp_weights`
// (same model, batch = block) or from `w` itself (block 1).
struct EigenvalueSolver {
  double tolerance = 1e-4;
  int max_iterations = 300;
  double hessian_eps = 1e-6;
  bool exact_hvp = false;
  unsigned long long seed = 42;
  int method = CDFT_EIGEN_RAYLEIGH_RITZ;
  int block = 1, max_basis = 32, check_interval = 4;
  cdft_eigen_config c() const {
    return {tolerance, max_iterations, hessian_eps, exact_hvp ? 1 : 0, seed, method, block, max_basis,
            check_interval};
  }
  EigenvalueResult solve(const functionals::Weights& w, const std::vector<double>& rho, double mu,
                         const std::vector<double>& initial_guess = {},
                         const functionals::Weights* hvp_weights = nullptr) const {
    DeviceVector d(rho);
    DeviceVector v(rho.size());
    if (initial_guess.size() == rho.size()) v.upload(initial_guess);
    cdft_eigen_config cfg = c();
    EigenvalueResult r;
    int it = 0, conv = 0;
    check(cdft_eigen_solve_ex(w.engine(), hvp_weights ? hvp_weights->engine() : nullptr, &cfg, d.get(), mu, v.get(),
                              initial_guess.size() == rho.size() ? 1 : 0, &r.eigenvalue, &it, &conv, nullptr));
    r.eigenvector = v.download();
    r.iterations = it;
    r.converged = conv != 0;
    return r;
  }
};

struct Result {
  std::vector<double> density, eigenvector;
  double grand_potential = 0.0, eigenvalue = 0.0;
  int outer_iterations = 0;
  bool converged = false;
  int eigen_iterations = 0, fire_steps = 0;  // summed over the outer iterations
};

// saddle_point.hpp:324-353 (same defaults)
struct Search {
  fire::Fire fire{1e-3, 1.0, 1e-8, 0.01, 1.1, 0.5, 1.0, 5, 20, 1e-4, 100000};
  EigenvalueSolver eigenvalue{1e-4, 300, 1e-6};
  minimization::Unbounded param{1e-18};
  double omega_tolerance = 1e-5, tolerance_start = 1e-3, tolerance_factor = 10.0;
  int max_outer_iterations = 20, eigenvalue_clear_count = 2;
  // FP64 defect correction of a mixed-precision search (see cdft_saddle_find_ex)
  const functionals::Weights* refine = nullptr;
  double refine_switch = 10.0;
  // product engine of a Lanczos eigen solve (batch = eigenvalue.block)
  const functionals::Weights* hvp_weights = nullptr;
  Result find(const physics::Model&, const functionals::Weights& w, const std::vector<double>& rho0, double mu,
              double target_mass) const {
    cdft_saddle_config cfg{fire.c(),        eigenvalue.c(),   param.rho_min,        omega_tolerance,
                           tolerance_start, tolerance_factor, max_outer_iterations, eigenvalue_clear_count};
    DeviceVector d(rho0);
    DeviceVector ev(rho0.size());
    double out[2] = {0.0, 0.0};
    int counts[3] = {0, 0, 0}, conv = 0;
    check(cdft_saddle_find_ex(w.engine(), refine ? refine->engine() : nullptr,
                              hvp_weights ? hvp_weights->engine() : nullptr, refine_switch, &cfg, d.get(), mu,
                              target_mass, ev.get(), out, counts, &conv, nullptr));
    Result r;
    r.density = d.download();
    r.eigenvector = ev.download();
    r.grand_potential = out[0];
    r.eigenvalue = out[1];
    r.outer_iterations = counts[0];
    r.eigen_iterations = counts[1];
    r.fire_steps = counts[2];
    r.converged = conv != 0;
    return r;
  }
};

}  // namespace saddle_point
}  // namespace algorithms

// ---------------------------------------------------------------- crystal

// types.hpp:52-71
enum class Structure : std::uint8_t { BCC = CDFT_BCC, FCC = CDFT_FCC, HCP = CDFT_HCP };
enum class Orientation : std::uint8_t {
  _001 = CDFT_ORIENT_001,
  _010 = CDFT_ORIENT_010,
  _100 = CDFT_ORIENT_100,
  _110 = CDFT_ORIENT_110,
  _101 = CDFT_ORIENT_101,
  _011 = CDFT_ORIENT_011,
  _111 = CDFT_ORIENT_111
};
enum class ExportFormat : std::uint8_t { XYZ = CDFT_EXPORT_XYZ, CSV = CDFT_EXPORT_CSV };

// types.hpp:73-83; positions are rows (x, y, z) with unit nearest-neighbour
// distance
static_assert(sizeof(std::array<double, 3>) == 3 * sizeof(double), "positions are passed as n x 3 doubles");
struct Lattice {
  Structure structure = Structure::FCC;
  Orientation orientation = Orientation::_001;
  std::vector<long> shape;
  std::array<double, 3> dimensions{};
  std::vector<std::array<double, 3>> positions;

  // crystal.cpp:247-255
  std::vector<std::array<double, 3>> scaled_positions(double dnn) const {
    auto out = positions;
    for (auto& p : out)
      for (double& x : p) x *= dnn;
    return out;
  }
  std::vector<std::array<double, 3>> scaled_positions(const std::array<double, 3>& box) const {
    auto out = positions;
    for (auto& p : out)
      for (int d = 0; d < 3; ++d) p[d] *= box[d] / dimensions[d];
    return out;
  }
  // crystal.cpp:257-279
  void export_to(const std::string& filename, ExportFormat format = ExportFormat::XYZ) const {
    check(cdft_lattice_export(positions.empty() ? nullptr : positions.data()->data(),
                              static_cast<long>(positions.size()), filename.c_str(), static_cast<int>(format)));
  }
};

// crystal.cpp:205-245
inline Lattice build_lattice(Structure structure, Orientation orientation, const std::vector<long>& shape = {1, 1, 1}) {
  if (shape.size() != 3) throw std::invalid_argument("Shape must have exactly 3 elements");
  long n = 0;
  check(cdft_lattice_size(static_cast<int>(structure), static_cast<int>(orientation), shape.data(), &n));
  Lattice l{structure, orientation, shape, {}, std::vector<std::array<double, 3>>(static_cast<std::size_t>(n))};
  check(cdft_build_lattice(static_cast<int>(structure), static_cast<int>(orientation), shape.data(),
                           l.positions.data()->data(), n, l.dimensions.data()));
  return l;
}

}  // namespace dft_b200
