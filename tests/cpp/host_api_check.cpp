// Drives the C++ host API (dft_b200.hpp) the way a user of the reference's
// C++ interface would: a one-species WhiteBear-II + Lennard-Jones model on a
// 16^3 grid (dx 0.25, kT 1, d 1, LJ sigma 1, epsilon 1, r_c 1.8), then
//   1. functionals::total with an external field and Functional::evaluate,
//   2. Minimizer::grand_potential (FIRE2 on the device),
//   3. Simulation::run, three integrating-factor DDFT steps at fixed dt,
//   4. Picard::solve (30 iterations), split_operator_step and
//      crank_nicholson_step, a Simulation with snapshots and a stop condition,
//   5. build_lattice and Lattice::export_to.
// Reads <dir>/rho.bin and <dir>/vext.bin (4096 doubles each); writes
// <dir>/force.bin, <dir>/min_rho.bin, <dir>/ddft_rho.bin, <dir>/picard_rho.bin,
// <dir>/split_rho.bin, <dir>/cn_rho.bin, <dir>/snap2_rho.bin,
// <dir>/lattice.xyz and prints the scalars as key=value lines.  The test that
// runs it compares them with the oracle.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "dft_b200/dft_b200.hpp"

namespace {

std::vector<double> read_doubles(const std::string& path, std::size_t n) {
  std::vector<double> v(n);
  std::ifstream f(path, std::ios::binary);
  if (!f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(sizeof(double) * n)))
    throw std::runtime_error("cannot read " + path);
  return v;
}

void write_doubles(const std::string& path, const std::vector<double>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(sizeof(double) * v.size()));
  if (!f) throw std::runtime_error("cannot write " + path);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 2) {
    std::cerr << "usage: host_api_check <dir>\n";
    return 2;
  }
  const std::string dir = argv[1];
  namespace d = dft_b200;
  try {
    d::physics::Model model;
    model.grid = d::make_grid(0.25, {4.0, 4.0, 4.0});
    model.species.push_back({"LJ", 1.0});
    model.interactions.push_back({0, 0, d::physics::make_lennard_jones(1.0, 1.0, 1.8)});
    model.temperature = 1.0;
    const std::size_t N = static_cast<std::size_t>(model.grid.total_points());

    const auto rho = read_doubles(dir + "/rho.bin", N);
    const auto vext = read_doubles(dir + "/vext.bin", N);

    // 1. total with a field, and the Functional wrapper without one
    d::functionals::Functional func(d::functionals::FMTModel::WhiteBearII(), model);
    d::functionals::State st;
    st.temperature = model.temperature;
    st.species.push_back({rho, vext, 0.7});
    const auto r = d::functionals::total(model, st, *func.weights);
    write_doubles(dir + "/force.bin", r.forces.at(0));
    const auto r0 = func.evaluate(rho, 0.7);
    std::printf("free_energy=%.17g\ngrand_potential=%.17g\n", r.free_energy, r.grand_potential);
    std::printf("free_energy_nofield=%.17g\ngrand_potential_nofield=%.17g\n", r0.free_energy, r0.grand_potential);
    std::printf("a_vdw=%.17g\n", func.weights->a_vdw().at(0));
    const auto cb = func.grand_potential_callback(0.7);
    std::printf("callback_omega=%.17g\n", cb({rho}).first);

    // 1b. total_stream: three states (with, without the field, scaled) equal to total on each
    {
      std::vector<d::functionals::State> states(3, st);
      states[1].species[0].external_field.clear();
      for (double& v : states[2].species[0].values) v *= 1.01;
      states[2].species[0].chemical_potential = 0.2;
      const auto rs = d::functionals::total_stream(model, states, *func.weights);
      int equal = rs.size() == 3;
      for (std::size_t i = 0; i < rs.size(); ++i) {
        const auto one = d::functionals::total(model, states[i], *func.weights);
        equal = equal && one.free_energy == rs[i].free_energy && one.grand_potential == rs[i].grand_potential &&
                one.forces == rs[i].forces;
      }
      std::printf("stream_equal=%d\n", equal);
    }

    // 1c. a mixed Weights anchored at rho, evaluated 1% off it
    {
      d::functionals::Weights wm(d::functionals::FMTModel::WhiteBearII(), model, CDFT_MIXED);
      wm.set_anchor(*func.weights, rho);
      d::functionals::State s1 = st;
      for (double& v : s1.species[0].values) v *= 1.01;
      const auto am = d::functionals::total(model, s1, wm);
      const auto a64 = d::functionals::total(model, s1, *func.weights);
      std::printf("anchor_dF=%.17g\n", std::abs(am.free_energy - a64.free_energy) / std::abs(a64.free_energy));
      wm.clear_anchor();
    }

    // 2. FIRE2 grand-potential minimisation
    d::algorithms::minimization::Minimizer mz;
    mz.fire.dt = 0.05;
    mz.fire.dt_max = 0.5;
    mz.fire.alpha_start = 0.01;
    mz.fire.f_alpha = 0.99;
    mz.fire.force_tolerance = 1e-10;
    mz.fire.max_steps = 4000;
    const auto m = mz.grand_potential(model, *func.weights, rho, 1.5);
    write_doubles(dir + "/min_rho.bin", m.densities.at(0));
    std::printf("min_converged=%d\nmin_iterations=%d\nmin_grand_potential=%.17g\n", m.converged ? 1 : 0,
                m.iterations, m.grand_potential);

    // 3. three DDFT steps at fixed dt
    d::algorithms::dynamics::Simulation sim;
    sim.step.dt = 2e-3;
    sim.step.dt_max = 2e-3;
    sim.step.fp_tolerance = 1e-10;
    sim.n_steps = 3;
    const auto s = sim.run({rho}, model.grid, *func.weights, 0.0);
    write_doubles(dir + "/ddft_rho.bin", s.densities.at(0));
    std::printf("ddft_energy=%.17g\nddft_time=%.17g\nmass_initial=%.17g\nmass_final=%.17g\n", s.energies.back(),
                s.times.back(), s.mass_initial, s.mass_final);

    // 4. Picard, the split-operator and Crank-Nicolson steps, snapshots
    d::algorithms::picard::Picard pc;
    pc.mixing = 0.1;
    pc.tolerance = 1e-14;
    pc.max_iterations = 30;
    const auto p = pc.solve({rho}, *func.weights, 1.5);
    write_doubles(dir + "/picard_rho.bin", p.densities.at(0));
    std::printf("picard_iterations=%d\npicard_omega=%.17g\n", p.iterations, p.grand_potential);
    d::algorithms::dynamics::StepConfig sc;
    sc.dt = 1e-3;
    sc.fp_tolerance = 1e-11;
    const auto so = d::algorithms::dynamics::split_operator_step({rho}, *func.weights, sc, 0.0);
    write_doubles(dir + "/split_rho.bin", so.densities.at(0));
    const auto cn = d::algorithms::dynamics::crank_nicholson_step({rho}, *func.weights, sc, 0.0);
    write_doubles(dir + "/cn_rho.bin", cn.densities.at(0));
    std::printf("split_energy=%.17g\ncn_energy=%.17g\n", so.energy, cn.energy);
    d::algorithms::dynamics::Simulation sim2 = sim;
    sim2.n_steps = 6;
    sim2.snapshot_interval = 2;
    sim2.log_interval = 0;
    sim2.stop_condition = [](int step, double, double) { return step == 5; };
    const auto s2 = sim2.run({rho}, model.grid, *func.weights, 0.0);
    std::printf("snapshots=%d\nsnapshot_last_step=%d\nrecorded=%d\n", static_cast<int>(s2.snapshots.size()),
                s2.snapshots.back().step, static_cast<int>(s2.times.size()));
    write_doubles(dir + "/snap2_rho.bin", s2.snapshots.at(1).densities.at(0));

    // 5. lattice
    const auto lat = d::build_lattice(d::Structure::HCP, d::Orientation::_010, {2, 1, 2});
    lat.export_to(dir + "/lattice.xyz", d::ExportFormat::XYZ);
    std::printf("lattice_sites=%d\nlattice_dim_y=%.17g\n", static_cast<int>(lat.positions.size()),
                lat.dimensions[1]);

    // 6. the reference's exception types
    try {
      d::make_grid(0.3, {1.0, 1.0, 1.0});
      std::printf("grid_error=none\n");
    } catch (const std::invalid_argument&) {
      std::printf("grid_error=invalid_argument\n");
    }
    try {
      d::functionals::State bad;
      bad.species.push_back({std::vector<double>(N - 1, 0.1), {}, 0.0});
      d::functionals::total(model, bad, *func.weights);
      std::printf("size_error=none\n");
    } catch (const std::invalid_argument&) {
      std::printf("size_error=invalid_argument\n");
    }
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
