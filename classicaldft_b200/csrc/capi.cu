// The extern "C" boundary (include/cdft_b200.h).  Every entry point catches
// all C++ exceptions and turns them into a status code plus a thread-local
// message, so nothing unwinds across the C ABI.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cdft_b200.h"
#include "drivers.cuh"
#include "engine.cuh"
#include "host_stream.cuh"
#include "physics.hpp"

struct cdft_engine {
  cdft::Engine* impl;
  cdft::Drivers* drivers;         // created on first driver call
  cdft::HostStream* host_stream;  // created on first cdft_total_stream call
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return CDFT_OK;
  } catch (const cdft::Error& e) {
    return fail(e.code(), e.what());
  } catch (const std::invalid_argument& e) {
    return fail(CDFT_ERR_INVALID, e.what());
  } catch (const std::bad_alloc& e) {
    return fail(CDFT_ERR_RUNTIME, std::string("allocation failed: ") + e.what());
  } catch (const std::exception& e) {
    return fail(CDFT_ERR_RUNTIME, e.what());
  } catch (...) {
    return fail(CDFT_ERR_RUNTIME, "unknown error");
  }
}

cdft::Potential to_potential(const cdft_potential* pot) {
  if (!pot) throw std::invalid_argument("potential is NULL");
  if (!(pot->sigma > 0.0)) throw std::invalid_argument("potential sigma must be positive");
  if (pot->type == CDFT_POT_WRDF && !(pot->r_cutoff > pot->sigma))
    throw std::invalid_argument("WRDF potential needs r_cutoff > sigma");
  return cdft::make_potential(pot->type, pot->sigma, pot->epsilon, pot->r_cutoff, pot->alpha);
}

void check_split(int split) {
  if (split != CDFT_SPLIT_WCA && split != CDFT_SPLIT_BH) throw std::invalid_argument("unknown split scheme");
}

}  // namespace

namespace cdft {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace cdft

extern "C" {

const char* cdft_last_error(void) { return g_last_error.c_str(); }

const char* cdft_version(void) { return "classicaldft_b200 0.1.0 (sm_100a)"; }

int cdft_potential_info(const cdft_potential* pot, double out[4]) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("out is NULL");
    cdft::Potential p = to_potential(pot);
    out[0] = p.epsilon_shift;
    out[1] = p.r_min;
    out[2] = p.v_min;
    out[3] = p.r_zero;
  });
}

int cdft_potential_attractive(const cdft_potential* pot, int split, const double* r, long n, double* out) {
  return guarded([&] {
    check_split(split);
    if (n < 0 || (n > 0 && (!r || !out))) throw std::invalid_argument("bad radius buffers");
    cdft::Potential p = to_potential(pot);
    for (long i = 0; i < n; ++i) out[i] = cdft::attractive(p, r[i], split);
  });
}

int cdft_hard_sphere_diameter(const cdft_potential* pot, double kT, int split, double* diameter) {
  return guarded([&] {
    check_split(split);
    if (!(kT > 0.0) || !diameter) throw std::invalid_argument("kT must be positive and diameter non-NULL");
    *diameter = cdft::hard_sphere_diameter(to_potential(pot), kT, split);
  });
}

int cdft_vdw_integral(const cdft_potential* pot, double kT, int split, double* value) {
  return guarded([&] {
    check_split(split);
    if (!(kT > 0.0) || !value) throw std::invalid_argument("kT must be positive and value non-NULL");
    *value = cdft::vdw_integral(to_potential(pot), kT, split);
  });
}

int cdft_interaction_weight(const long shape[3], double dx, const cdft_potential* pot, int split, int scheme,
                            double kT, double* weight_out, double* a_vdw) {
  return guarded([&] {
    check_split(split);
    if (!shape || shape[0] <= 0 || shape[1] <= 0 || shape[2] <= 0) throw std::invalid_argument("bad grid shape");
    if (!(dx > 0.0) || !(kT > 0.0)) throw std::invalid_argument("dx and kT must be positive");
    if (scheme < CDFT_WEIGHT_ZERO || scheme > CDFT_WEIGHT_GAUSS_F) throw std::invalid_argument("unknown weight scheme");
    if (!weight_out) throw std::invalid_argument("weight_out is NULL");
    double a = cdft::interaction_weight(shape, dx, to_potential(pot), split, scheme, kT, weight_out);
    if (a_vdw) *a_vdw = a;
  });
}

}  // extern "C"

namespace {

// The grid / species / FMT part of an engine spec, validated.
cdft::EngineSpec base_spec(const long shape[3], double dx, int n_species, const double* diameters, int fmt_model,
                           double esfmt_A, double esfmt_B, int n_interactions, const void* interactions, int precision,
                           int batch) {
  if (!shape) throw std::invalid_argument("shape is NULL");
  if (n_species < 1 || !diameters) throw std::invalid_argument("need at least one species diameter");
  if (n_interactions < 0 || (n_interactions > 0 && !interactions)) throw std::invalid_argument("interactions is NULL");
  if (batch < 1 || batch > CDFT_MAX_BATCH) throw std::invalid_argument("batch must be in [1, 64]");
  if (shape[0] <= 0 || shape[1] <= 0 || shape[2] <= 0) throw std::invalid_argument("grid dimensions must be positive");
  cdft::EngineSpec spec;
  for (int d = 0; d < 3; ++d) spec.shape[d] = shape[d];
  spec.dx = dx;
  spec.diameters.assign(diameters, diameters + n_species);
  spec.model = fmt_model;
  spec.esfmt_A = esfmt_A;
  spec.esfmt_B = esfmt_B;
  spec.precision = precision;
  spec.batch = batch;
  return spec;
}

void make_engine(cdft_engine** out, const cdft::EngineSpec& spec) {
  auto* e = new cdft_engine{nullptr, nullptr, nullptr};
  try {
    e->impl = new cdft::Engine(spec);
  } catch (...) {
    delete e;
    throw;
  }
  *out = e;
}

}  // namespace

extern "C" {

int cdft_create_batch(cdft_engine** out, const long shape[3], double dx, int n_species, const double* diameters,
                      int fmt_model, double esfmt_A, double esfmt_B, int n_interactions,
                      const cdft_interaction* interactions, int precision, int batch) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("out is NULL");
    *out = nullptr;
    cdft::EngineSpec spec = base_spec(shape, dx, n_species, diameters, fmt_model, esfmt_A, esfmt_B, n_interactions,
                                      interactions, precision, batch);
    const long long N = (long long)shape[0] * shape[1] * shape[2];
    for (int m = 0; m < n_interactions; ++m) {
      cdft::InteractionSpec is;
      is.species_i = interactions[m].species_i;
      is.species_j = interactions[m].species_j;
      if (!interactions[m].weight_real) throw std::invalid_argument("interaction weight_real is NULL");
      is.weight_real.assign(interactions[m].weight_real, interactions[m].weight_real + N);
      is.a_vdw = interactions[m].a_vdw;
      spec.interactions.push_back(std::move(is));
    }
    make_engine(out, spec);
  });
}

int cdft_create_model(cdft_engine** out, const long shape[3], double dx, int n_species, const double* diameters,
                      int fmt_model, double esfmt_A, double esfmt_B, int n_interactions,
                      const cdft_model_interaction* interactions, double kT, int precision, int batch) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("out is NULL");
    *out = nullptr;
    if (!(kT > 0.0)) throw std::invalid_argument("the temperature must be positive");
    cdft::EngineSpec spec = base_spec(shape, dx, n_species, diameters, fmt_model, esfmt_A, esfmt_B, n_interactions,
                                      interactions, precision, batch);
    for (int m = 0; m < n_interactions; ++m) {
      const cdft_model_interaction& mi = interactions[m];
      check_split(mi.split);
      if (mi.scheme < CDFT_WEIGHT_ZERO || mi.scheme > CDFT_WEIGHT_GAUSS_F)
        throw std::invalid_argument("unknown weight scheme");
      cdft::InteractionSpec is;
      is.species_i = mi.species_i;
      is.species_j = mi.species_j;
      is.on_device = true;
      is.potential = to_potential(&mi.potential);
      is.split = mi.split;
      is.scheme = mi.scheme;
      is.kT = kT;
      spec.interactions.push_back(std::move(is));
    }
    make_engine(out, spec);
  });
}

int cdft_create(cdft_engine** out, const long shape[3], double dx, int n_species, const double* diameters,
                int fmt_model, double esfmt_A, double esfmt_B, int n_interactions,
                const cdft_interaction* interactions, int precision) {
  return cdft_create_batch(out, shape, dx, n_species, diameters, fmt_model, esfmt_A, esfmt_B, n_interactions,
                           interactions, precision, 1);
}

int cdft_engine_batch(const cdft_engine* engine, int* batch) {
  return guarded([&] {
    if (!engine || !batch) throw std::invalid_argument("engine or batch is NULL");
    *batch = engine->impl->batch();
  });
}

int cdft_engine_bulk_model(const cdft_engine* engine, cdft_bulk_model* out) {
  return guarded([&] {
    if (!engine || !out) throw std::invalid_argument("engine or out is NULL");
    const cdft::EvalParams& p = engine->impl->params();
    *out = cdft_bulk_model{};
    out->n_species = p.S;
    for (int s = 0; s < p.S; ++s) out->diameters[s] = 2.0 * p.R[s];
    out->fmt_model = p.model;
    out->esfmt_A = p.A;
    out->esfmt_B = p.B;
    out->n_interactions = p.M;
    for (int m = 0; m < p.M; ++m) out->interactions[m] = {p.mf_i[m], p.mf_j[m], engine->impl->a_vdw(m)};
  });
}

int cdft_destroy(cdft_engine* engine) {
  return guarded([&] {
    if (!engine) return;
    delete engine->host_stream;
    delete engine->drivers;
    delete engine->impl;
    delete engine;
  });
}

int cdft_engine_info(const cdft_engine* engine, long long info[8]) {
  return guarded([&] {
    if (!engine || !info) throw std::invalid_argument("engine or info is NULL");
    const cdft::Engine& e = *engine->impl;
    info[0] = e.points();
    info[1] = e.modes();
    info[2] = e.species();
    info[3] = e.params().n_chan;
    info[4] = e.params().L.n_deriv;
    info[5] = e.precision();
    info[6] = e.kernels_per_eval();
    info[7] = (long long)e.scratch_bytes();
  });
}

int cdft_engine_a_vdw(const cdft_engine* engine, int m, double* a_vdw) {
  return guarded([&] {
    if (!engine || !a_vdw) throw std::invalid_argument("engine or a_vdw is NULL");
    if (m < 0 || m >= engine->impl->params().M) throw std::invalid_argument("interaction index out of range");
    *a_vdw = engine->impl->a_vdw(m);
  });
}

int cdft_total(cdft_engine* engine, const double* rho, const double* vext, const double* mu, double* force,
               double* scalars) {
  return guarded([&] {
    if (!engine || !rho || !mu) throw std::invalid_argument("engine, rho and mu are required");
    cdft::Engine& e = *engine->impl;
    const size_t bytes = sizeof(double) * e.batch() * e.species() * e.points();
    cudaStream_t st = e.stream();
    CDFT_CUDA(cudaMemcpyAsync(e.host_rho(), rho, bytes, cudaMemcpyHostToDevice, st));
    if (vext) CDFT_CUDA(cudaMemcpyAsync(e.host_vext(), vext, bytes, cudaMemcpyHostToDevice, st));
    e.evaluate(e.host_rho(), vext ? e.host_vext() : nullptr, mu, e.host_force(), e.host_scalars(), st);
    if (force) CDFT_CUDA(cudaMemcpyAsync(force, e.host_force(), bytes, cudaMemcpyDeviceToHost, st));
    std::vector<double> tmp((size_t)e.batch() * CDFT_SCALAR_COUNT);
    CDFT_CUDA(cudaMemcpyAsync(tmp.data(), e.host_scalars(), sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost, st));
    CDFT_CUDA(cudaStreamSynchronize(st));
    if (e.take_error(st)) throw cdft::Error(CDFT_ERR_RUNTIME, "evaluation aborted: a bounded device wait timed out");
    if (scalars) std::memcpy(scalars, tmp.data(), sizeof(double) * tmp.size());
  });
}

int cdft_total_stream(cdft_engine* engine, int count, const double* const* rho, const double* const* vext,
                      const double* mu, double* const* force, double* scalars) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    if (!engine->host_stream) engine->host_stream = new cdft::HostStream(*engine->impl);
    engine->host_stream->run(count, rho, vext, mu, force, scalars);
  });
}

int cdft_total_device(cdft_engine* engine, const double* rho, const double* vext, const double* mu, double* force,
                      double* scalars, void* stream) {
  return guarded([&] {
    if (!engine || !rho || !mu || !force || !scalars)
      throw std::invalid_argument("engine, rho, mu, force and scalars are required");
    engine->impl->evaluate(rho, vext, mu, force, scalars, static_cast<cudaStream_t>(stream));
  });
}

int cdft_engine_stage_timing(cdft_engine* engine, int on) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    engine->impl->set_stage_timing(on != 0);
  });
}

int cdft_engine_stage_times(cdft_engine* engine, double ms[CDFT_STAGE_COUNT], long long* evaluations) {
  return guarded([&] {
    if (!engine || !ms) throw std::invalid_argument("engine and ms are required");
    static_assert(CDFT_STAGE_COUNT == cdft::Engine::kStages, "stage count");
    const long long n = engine->impl->take_stage_times(ms);
    if (evaluations) *evaluations = n;
  });
}

int cdft_engine_set_transforms(cdft_engine* engine, int transforms) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    if (transforms != CDFT_TRANSFORMS_CUFFT && transforms != CDFT_TRANSFORMS_FUSED)
      throw std::invalid_argument("unknown transform implementation");
    engine->impl->set_fused(transforms == CDFT_TRANSFORMS_FUSED);
  });
}

int cdft_engine_set_plane_chunks(cdft_engine* engine, int chunks) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    static_assert(CDFT_MAX_PLANE_CHUNKS == cdft::Engine::kMaxChunks, "chunk limit");
    engine->impl->set_chunks(chunks);
  });
}

int cdft_set_step_graphs(int on) {
  return guarded([&] { cdft::set_step_graphs(on != 0); });
}

int cdft_step_graphs(int* on) {
  return guarded([&] {
    if (!on) throw std::invalid_argument("on is NULL");
    *on = cdft::step_graphs() ? 1 : 0;
  });
}

int cdft_engine_autotune(cdft_engine* engine, const double* rho, const double* vext, const double* mu,
                         void* stream, int reps, int* chunks, double* ms) {
  return guarded([&] {
    if (!engine || !rho) throw std::invalid_argument("engine and rho are required");
    if (reps < 1) throw std::invalid_argument("autotune: reps must be positive");
    using E = cdft::Engine;
    double all[2 * E::kPointwiseVariants * E::kMaxChunks * E::kSpreads];
    int v = 0, tq = 16, d = 0;
    const int k = engine->impl->autotune(rho, vext, mu, static_cast<cudaStream_t>(stream), reps, all, &v, &tq, &d);
    if (chunks) *chunks = k;
    const int ti = tq == 32 ? 1 : 0;
    if (ms)  // per chunk count: the best spread at the kept tile and variant
      for (int c = 0; c < E::kMaxChunks; ++c) {
        double best = 0.0;
        for (int di = 0; di < E::kSpreads; ++di) {
          const double t = all[((ti * E::kPointwiseVariants + v) * E::kMaxChunks + c) * E::kSpreads + di];
          if (t > 0.0 && (best == 0.0 || t < best)) best = t;
        }
        ms[c] = best;
      }
  });
}

int cdft_engine_autotune_ex(cdft_engine* engine, const double* rho, const double* vext, const double* mu,
                            void* stream, int reps, int choice[4], double* ms) {
  return guarded([&] {
    if (!engine || !rho) throw std::invalid_argument("engine and rho are required");
    if (reps < 1) throw std::invalid_argument("autotune: reps must be positive");
    int v = 0, tq = 0, d = 0;
    const int k = engine->impl->autotune(rho, vext, mu, static_cast<cudaStream_t>(stream), reps, ms, &v, &tq, &d);
    if (choice) {
      choice[0] = k;
      choice[1] = v;
      choice[2] = tq;
      choice[3] = d;
    }
  });
}

int cdft_engine_set_anchor(cdft_engine* engine, cdft_engine* fp64_engine, const double* rho_anchor, void* stream) {
  return guarded([&] {
    if (!engine || !fp64_engine || !rho_anchor)
      throw std::invalid_argument("anchor: engine, the FP64 engine and rho_anchor are required");
    engine->impl->set_anchor(*fp64_engine->impl, rho_anchor, static_cast<cudaStream_t>(stream));
  });
}

int cdft_engine_set_anchor_host(cdft_engine* engine, cdft_engine* fp64_engine, const double* rho_anchor) {
  return guarded([&] {
    if (!engine || !fp64_engine || !rho_anchor)
      throw std::invalid_argument("anchor: engine, the FP64 engine and rho_anchor are required");
    cdft::Engine& e = *engine->impl;
    const size_t bytes = sizeof(double) * e.batch() * e.species() * e.points();
    cudaStream_t st = e.stream();
    CDFT_CUDA(cudaMemcpyAsync(e.host_rho(), rho_anchor, bytes, cudaMemcpyHostToDevice, st));
    e.set_anchor(*fp64_engine->impl, e.host_rho(), st);
  });
}

int cdft_engine_set_dependent_launch(cdft_engine* engine, int on, int* was) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    if (was) *was = engine->impl->dependent_launch() ? 1 : 0;
    if (on >= 0) engine->impl->set_dependent_launch(on != 0);
  });
}

int cdft_engine_clear_anchor(cdft_engine* engine) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    engine->impl->clear_anchor();
  });
}

int cdft_engine_anchored(const cdft_engine* engine, int* anchored) {
  return guarded([&] {
    if (!engine || !anchored) throw std::invalid_argument("engine and anchored are required");
    *anchored = engine->impl->anchored() ? 1 : 0;
  });
}

int cdft_engine_set_pointwise_spread(cdft_engine* engine, int spread) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    engine->impl->set_pw_spread(spread);
  });
}

int cdft_engine_pointwise_spread(const cdft_engine* engine, int* spread) {
  return guarded([&] {
    if (!engine || !spread) throw std::invalid_argument("engine and spread are required");
    *spread = engine->impl->pw_spread();
  });
}

int cdft_engine_set_plane_width(cdft_engine* engine, int wide) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    engine->impl->set_plane_width(wide);
  });
}

int cdft_engine_plane_width(const cdft_engine* engine, int* wide) {
  return guarded([&] {
    if (!engine || !wide) throw std::invalid_argument("engine and wide are required");
    *wide = engine->impl->plane_width();
  });
}

int cdft_engine_set_column_tile(cdft_engine* engine, int tile) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    engine->impl->set_col_tile(tile);
  });
}

int cdft_engine_column_tile(const cdft_engine* engine, int* tile) {
  return guarded([&] {
    if (!engine || !tile) throw std::invalid_argument("engine and tile are required");
    *tile = engine->impl->col_tile();
  });
}

int cdft_engine_set_pointwise(cdft_engine* engine, int variant) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    engine->impl->set_pointwise(variant);
  });
}

int cdft_engine_pointwise(const cdft_engine* engine, int* variant, int* available) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    if (variant) *variant = engine->impl->pointwise();
    if (available) *available = engine->impl->pointwise_one_species() ? 1 : 0;
  });
}

int cdft_engine_transforms(const cdft_engine* engine, int* transforms, int* fused_available) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    if (transforms) *transforms = engine->impl->fused() ? CDFT_TRANSFORMS_FUSED : CDFT_TRANSFORMS_CUFFT;
    if (fused_available) *fused_available = engine->impl->fusable() ? 1 : 0;
  });
}

int cdft_engine_status(cdft_engine* engine, void* stream) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is NULL");
    if (engine->impl->take_error(static_cast<cudaStream_t>(stream)))
      throw cdft::Error(CDFT_ERR_RUNTIME, "a bounded device wait timed out in an earlier call");
  });
}

namespace {

cdft::Drivers& drivers_of(cdft_engine* e, bool batched = false) {
  if (!e) throw std::invalid_argument("engine is NULL");
  if (!batched && e->impl->batch() != 1) throw std::invalid_argument("the drivers need an engine with batch 1");
  if (!e->drivers) e->drivers = new cdft::Drivers(*e->impl);
  return *e->drivers;
}

cdft::FireParams to_fire(const cdft_fire_params& f) {
  cdft::FireParams p;
  p.dt = f.dt;
  p.dt_max = f.dt_max;
  p.dt_min = f.dt_min;
  p.alpha_start = f.alpha_start;
  p.f_inc = f.f_inc;
  p.f_dec = f.f_dec;
  p.f_alpha = f.f_alpha;
  p.n_delay = f.n_delay;
  p.max_uphill = f.max_uphill;
  p.force_tolerance = f.force_tolerance;
  p.max_steps = f.max_steps;
  if (!(p.dt > 0.0) || p.max_steps < 0) throw std::invalid_argument("FIRE: dt must be positive, max_steps >= 0");
  return p;
}

cdft::Drivers::EigenConfig to_eigen(const cdft_eigen_config& c) {
  cdft::Drivers::EigenConfig e;
  e.tolerance = c.tolerance;
  e.max_iterations = c.max_iterations;
  e.hessian_eps = c.hessian_eps;
  e.exact_hvp = c.exact_hvp;
  e.seed = c.seed;
  e.method = c.method;
  if (e.method != CDFT_EIGEN_RAYLEIGH_RITZ && e.method != CDFT_EIGEN_LANCZOS)
    throw std::invalid_argument("eigen: unknown method");
  e.block = c.block > 0 ? c.block : 1;
  e.max_basis = c.max_basis > 0 ? c.max_basis : 32;
  e.check_interval = c.check_interval > 0 ? c.check_interval : 4;
  return e;
}

}  // namespace

namespace {
cdft::FireConfig to_fire_config(const cdft_minimizer_config* cfg) {
  cdft::FireConfig fc;
  fc.fire = to_fire(cfg->fire);
  fc.mode = cfg->mode;
  if (fc.mode < CDFT_MIN_GRAND_POTENTIAL || fc.mode > CDFT_MIN_SADDLE) throw std::invalid_argument("unknown mode");
  fc.param = cfg->parametrization;
  fc.rho_min = cfg->rho_min;
  fc.rho_max = cfg->rho_max;
  fc.homogeneous_boundary = cfg->homogeneous_boundary != 0;
  fc.mu = cfg->chemical_potential;
  fc.target_mass = cfg->target_mass;
  fc.boundary_mass = cfg->boundary_mass;
  fc.use_monitor = cfg->use_monitor != 0;
  fc.check_interval = cfg->check_interval > 0 ? cfg->check_interval : 25;
  fc.vext = cfg->external_field;
  return fc;
}

void to_result(const cdft::FireResult& r, cdft_minimizer_result* result) {
  result->free_energy = r.free_energy;
  result->grand_potential = r.grand_potential;
  result->rms_force = r.rms_force;
  result->iterations = r.iterations;
  result->converged = r.converged ? 1 : 0;
  result->uphill_error = r.uphill_error ? 1 : 0;
}
}  // namespace

int cdft_minimize(cdft_engine* engine, const cdft_minimizer_config* cfg, double* rho, const double* direction,
                  cdft_engine* refine, double refine_switch, cdft_minimizer_result* result, void* stream) {
  return guarded([&] {
    if (!cfg || !rho || !result) throw std::invalid_argument("cfg, rho and result are required");
    cdft::Drivers& d = drivers_of(engine);
    if (refine && refine->impl->batch() != 1) throw std::invalid_argument("the refine engine needs batch 1");
    cdft::FireConfig fc = to_fire_config(cfg);
    cdft::FireResult r = d.fire_minimize(fc, rho, direction, static_cast<cudaStream_t>(stream),
                                         refine ? refine->impl : nullptr, refine_switch);
    to_result(r, result);
    if (r.uphill_error) throw cdft::Error(CDFT_ERR_RUNTIME, "fire::step: exceeded max uphill steps");
  });
}

int cdft_minimize_batch(cdft_engine* engine, const cdft_minimizer_config* cfg, const double* mu,
                        const double* target_mass, double* rho, cdft_engine* refine, double refine_switch,
                        cdft_minimizer_result* results, void* stream) {
  return guarded([&] {
    if (!cfg || !mu || !rho || !results) throw std::invalid_argument("cfg, mu, rho and results are required");
    cdft::Drivers& d = drivers_of(engine, true);
    if (cfg->mode == CDFT_MIN_SADDLE) throw std::invalid_argument("cdft_minimize_batch: no saddle mode");
    cdft::FireConfig fc = to_fire_config(cfg);
    std::vector<cdft::FireResult> r = d.fire_minimize_batch(fc, mu, target_mass, rho, static_cast<cudaStream_t>(stream),
                                                            refine ? refine->impl : nullptr, refine_switch);
    for (size_t b = 0; b < r.size(); ++b) to_result(r[b], results + b);
  });
}

namespace {
cdft::Drivers::DDFTConfig to_ddft(const cdft_ddft_config& c, double mu) {
  cdft::Drivers::DDFTConfig d;
  d.dt = c.dt;
  d.diffusion = c.diffusion_coefficient;
  d.min_density = c.min_density;
  d.dt_max = c.dt_max;
  d.fp_tolerance = c.fp_tolerance;
  d.fp_max_iterations = c.fp_max_iterations;
  d.mu = mu;
  if (!(d.dt > 0.0)) throw std::invalid_argument("DDFT: dt must be positive");
  return d;
}
}  // namespace

int cdft_minimize_group(int n_members, const cdft_group_member* members, const cdft_minimizer_config* cfg,
                        void* stream) {
  return guarded([&] {
    if (n_members < 1 || !members || !cfg) throw std::invalid_argument("members and cfg are required");
    cdft::FireConfig fc = to_fire_config(cfg);
    std::vector<cdft::GroupMember> g(n_members);
    for (int m = 0; m < n_members; ++m) {
      const cdft_group_member& c = members[m];
      if (!c.engine || !c.results) throw std::invalid_argument("every member needs an engine and results");
      g[m].drivers = &drivers_of(c.engine, true);
      g[m].mu = c.mu;
      g[m].mass = c.target_mass;
      g[m].rho = c.rho;
      g[m].refine = c.refine ? c.refine->impl : nullptr;
      g[m].refine_switch = c.refine_switch > 0.0 ? c.refine_switch : 10.0;
    }
    const std::vector<std::vector<cdft::FireResult>> r =
        cdft::fire_minimize_group(g, fc, static_cast<cudaStream_t>(stream));
    for (int m = 0; m < n_members; ++m)
      for (size_t b = 0; b < r[m].size(); ++b) {
        cdft_minimizer_result& o = members[m].results[b];
        o.free_energy = r[m][b].free_energy;
        o.grand_potential = r[m][b].grand_potential;
        o.rms_force = r[m][b].rms_force;
        o.iterations = r[m][b].iterations;
        o.converged = r[m][b].converged ? 1 : 0;
        o.uphill_error = r[m][b].uphill_error ? 1 : 0;
      }
  });
}


int cdft_ddft_step(cdft_engine* engine, cdft_ddft_config* cfg, double chemical_potential, double* rho,
                   double* energy, int* fp_iterations, void* stream) {
  return guarded([&] {
    if (!cfg || !rho) throw std::invalid_argument("cfg and rho are required");
    cdft::Drivers& d = drivers_of(engine);
    cdft::Drivers::DDFTConfig dc = to_ddft(*cfg, chemical_potential);
    const double e = d.ddft_step(dc, rho, static_cast<cudaStream_t>(stream), fp_iterations);
    cfg->dt = dc.dt;
    if (energy) *energy = e;
  });
}

int cdft_ddft_set_refine(cdft_engine* engine, cdft_engine* refine, int iterations) {
  return guarded([&] {
    if (!engine) throw std::invalid_argument("engine is required");
    drivers_of(engine).set_ddft_refine(refine ? refine->impl : nullptr, iterations);
  });
}

int cdft_ddft_last_step(cdft_engine* engine, int info[4], double* refine_deviation) {
  return guarded([&] {
    if (!engine || !info) throw std::invalid_argument("engine and info are required");
    const cdft::Drivers::DDFTStepInfo& i = drivers_of(engine).last_ddft_step();
    info[0] = i.fp_iterations;
    info[1] = i.restarts;
    info[2] = i.status;
    info[3] = i.device_loop;
    if (refine_deviation) *refine_deviation = i.refine_deviation;
  });
}

int cdft_ddft_run(cdft_engine* engine, cdft_ddft_config* cfg, double chemical_potential, int n_steps, double* rho,
                  double* times, double* energies, void* stream) {
  return guarded([&] {
    if (!cfg || !rho || n_steps < 0) throw std::invalid_argument("cfg, rho and n_steps >= 0 are required");
    cdft::Drivers& d = drivers_of(engine);
    cdft::Drivers::DDFTConfig dc = to_ddft(*cfg, chemical_potential);
    d.ddft_run(dc, n_steps, rho, times, energies, 0, nullptr, nullptr, nullptr, nullptr,
               static_cast<cudaStream_t>(stream));
    cfg->dt = dc.dt;
  });
}

int cdft_ddft_split_step(cdft_engine* engine, const cdft_ddft_config* cfg, double chemical_potential, double* rho,
                         double* energy, void* stream) {
  return guarded([&] {
    if (!cfg || !rho) throw std::invalid_argument("cfg and rho are required");
    cdft::Drivers& d = drivers_of(engine);
    const double e = d.ddft_split_step(to_ddft(*cfg, chemical_potential), rho, static_cast<cudaStream_t>(stream));
    if (energy) *energy = e;
  });
}

int cdft_ddft_cn_step(cdft_engine* engine, const cdft_ddft_config* cfg, double chemical_potential, double* rho,
                      double* energy, int* fp_iterations, void* stream) {
  return guarded([&] {
    if (!cfg || !rho) throw std::invalid_argument("cfg and rho are required");
    cdft::Drivers& d = drivers_of(engine);
    const double e =
        d.ddft_cn_step(to_ddft(*cfg, chemical_potential), rho, static_cast<cudaStream_t>(stream), fp_iterations);
    if (energy) *energy = e;
  });
}

int cdft_ddft_simulate(cdft_engine* engine, cdft_ddft_config* cfg, double chemical_potential, int n_steps,
                       double* rho, double* times, double* energies, int snapshot_interval, double* snapshots,
                       int* snapshot_steps, int snapshot_capacity, int* snapshot_count,
                       const unsigned char* reservoir_mask, double reservoir_density, cdft_ddft_stop_fn stop,
                       void* user, int* steps_done, void* stream) {
  return guarded([&] {
    if (!cfg || !rho || n_steps < 0) throw std::invalid_argument("cfg, rho and n_steps >= 0 are required");
    if (snapshot_interval < 0 || snapshot_capacity < 0 || (snapshot_capacity > 0 && !snapshots))
      throw std::invalid_argument("snapshots: interval >= 0, and a buffer for a positive capacity");
    cdft::Drivers& d = drivers_of(engine);
    cdft::Drivers::DDFTConfig dc = to_ddft(*cfg, chemical_potential);
    cdft::Drivers::SnapshotSink sink;
    sink.host = snapshots;
    sink.steps = snapshot_steps;
    sink.capacity = snapshot_capacity;
    int done = 0;
    try {
      cdft::Drivers::Reservoir res;
      res.mask = reservoir_mask;
      res.density = reservoir_density;
      done = d.ddft_run(dc, n_steps, rho, times, energies, snapshot_interval, &sink, stop, user, &res,
                        static_cast<cudaStream_t>(stream));
    } catch (...) {
      if (snapshot_count) *snapshot_count = sink.count;
      throw;
    }
    cfg->dt = dc.dt;
    if (snapshot_count) *snapshot_count = sink.count;
    if (steps_done) *steps_done = done;
  });
}

int cdft_picard(cdft_engine* engine, const cdft_picard_config* cfg, const double* mu, const double* target_mass,
                const double* background, double* rho, cdft_picard_result* results, void* stream) {
  return guarded([&] {
    if (!cfg || !mu || !rho || !results) throw std::invalid_argument("cfg, mu, rho and results are required");
    if (!(cfg->mixing > 0.0) || cfg->max_iterations < 0)
      throw std::invalid_argument("picard: mixing > 0 and max_iterations >= 0 are required");
    cdft::Drivers& d = drivers_of(engine, true);
    cdft::Drivers::PicardConfig pc;
    pc.mixing = cfg->mixing;
    pc.min_density = cfg->min_density;
    pc.tolerance = cfg->tolerance;
    pc.constraint_min_density = cfg->constraint_min_density;
    pc.max_iterations = cfg->max_iterations;
    pc.check_interval = cfg->check_interval > 0 ? cfg->check_interval : 25;
    std::vector<cdft::Drivers::PicardResult> r =
        d.picard(pc, mu, target_mass, background, rho, static_cast<cudaStream_t>(stream));
    for (size_t b = 0; b < r.size(); ++b) {
      results[b].grand_potential = r[b].grand_potential;
      results[b].residual = r[b].residual;
      results[b].iterations = r[b].iterations;
      results[b].converged = r[b].converged ? 1 : 0;
    }
  });
}

int cdft_hvp(cdft_engine* engine, const double* rho, const double* v, double chemical_potential, int boundary,
             double* hv, void* stream) {
  return guarded([&] {
    if (!rho || !v || !hv) throw std::invalid_argument("rho, v and hv are required");
    if (engine && engine->impl->species() != 1) {
      double mu[4] = {chemical_potential, chemical_potential, chemical_potential, chemical_potential};
      engine->impl->hvp(rho, v, mu, hv, static_cast<cudaStream_t>(stream));
      return;
    }
    drivers_of(engine).hvp_exact(rho, v, hv, chemical_potential, boundary, static_cast<cudaStream_t>(stream));
  });
}

int cdft_hvp_fd(cdft_engine* engine, const double* rho, const double* force_at_rho, const double* v,
                double chemical_potential, double eps, int boundary, double* hv, void* stream) {
  return guarded([&] {
    if (!rho || !force_at_rho || !v || !hv || !(eps > 0.0)) throw std::invalid_argument("bad HVP arguments");
    drivers_of(engine).hvp_fd(rho, force_at_rho, v, hv, eps, chemical_potential, boundary,
                              static_cast<cudaStream_t>(stream));
  });
}

int cdft_eigen_solve(cdft_engine* engine, const cdft_eigen_config* cfg, const double* rho, double chemical_potential,
                     double* vec, int use_guess, double* eigenvalue, int* iterations, int* converged, void* stream) {
  return guarded([&] {
    if (!cfg || !rho || !vec) throw std::invalid_argument("cfg, rho and vec are required");
    cdft::Drivers::EigenResult r = drivers_of(engine).eigen_solve(to_eigen(*cfg), rho, chemical_potential, vec,
                                                                  use_guess != 0, static_cast<cudaStream_t>(stream));
    if (eigenvalue) *eigenvalue = r.eigenvalue;
    if (iterations) *iterations = r.iterations;
    if (converged) *converged = r.converged ? 1 : 0;
  });
}

int cdft_eigen_solve_ex(cdft_engine* engine, cdft_engine* hvp_engine, const cdft_eigen_config* cfg,
                        const double* rho, double chemical_potential, double* vec, int use_guess, double* eigenvalue,
                        int* iterations, int* converged, void* stream) {
  return guarded([&] {
    if (!cfg || !rho || !vec) throw std::invalid_argument("cfg, rho and vec are required");
    cdft::Engine* he = hvp_engine ? hvp_engine->impl : nullptr;
    cdft::Drivers::EigenResult r = drivers_of(engine).eigen_solve(to_eigen(*cfg), rho, chemical_potential, vec,
                                                                  use_guess != 0, static_cast<cudaStream_t>(stream),
                                                                  he);
    if (eigenvalue) *eigenvalue = r.eigenvalue;
    if (iterations) *iterations = r.iterations;
    if (converged) *converged = r.converged ? 1 : 0;
  });
}

int cdft_saddle_find(cdft_engine* engine, const cdft_saddle_config* cfg, double* rho, double chemical_potential,
                     double target_mass, double* eigvec, double out[2], int* outer_iterations, int* converged,
                     void* stream) {
  int counts[3] = {0, 0, 0};
  const int st = cdft_saddle_find_ex(engine, nullptr, nullptr, 10.0, cfg, rho, chemical_potential, target_mass, eigvec,
                                     out, counts, converged, stream);
  if (st == CDFT_OK && outer_iterations) *outer_iterations = counts[0];
  return st;
}

int cdft_saddle_find_ex(cdft_engine* engine, cdft_engine* refine, cdft_engine* hvp_engine, double refine_switch,
                        const cdft_saddle_config* cfg, double* rho, double chemical_potential, double target_mass,
                        double* eigvec, double out[2], int counts[3], int* converged, void* stream) {
  return guarded([&] {
    if (!cfg || !rho || !eigvec) throw std::invalid_argument("cfg, rho and eigvec are required");
    if (refine && refine->impl->precision() != cdft::kFP64)
      throw std::invalid_argument("saddle: the refine engine must be FP64");
    cdft::Drivers::SaddleConfig sc;
    sc.fire = to_fire(cfg->fire);
    sc.eigen = to_eigen(cfg->eigen);
    sc.rho_min = cfg->rho_min;
    sc.omega_tolerance = cfg->omega_tolerance;
    sc.tolerance_start = cfg->tolerance_start;
    sc.tolerance_factor = cfg->tolerance_factor;
    sc.max_outer_iterations = cfg->max_outer_iterations;
    sc.eigenvalue_clear_count = cfg->eigenvalue_clear_count;
    cdft::Drivers::SaddleResult r = drivers_of(engine).saddle_find(
        sc, rho, chemical_potential, target_mass, eigvec, static_cast<cudaStream_t>(stream),
        refine ? refine->impl : nullptr, hvp_engine ? hvp_engine->impl : nullptr, refine_switch);
    if (out) {
      out[0] = r.grand_potential;
      out[1] = r.eigenvalue;
    }
    if (counts) {
      counts[0] = r.outer_iterations;
      counts[1] = r.eigen_iterations;
      counts[2] = r.fire_steps;
    }
    if (converged) *converged = r.converged ? 1 : 0;
  });
}

}  // extern "C"
