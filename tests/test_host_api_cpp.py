"""The C++ host API (include/dft_b200/dft_b200.hpp): the check program in
tests/cpp is compiled with g++ against the header and libcdft_b200.so (CPU
test), then run on the GPU and compared with the oracle: F and Omega to
1e-12 relative and forces to 1e-11 of their max (the tolerances of the other
FP64 parity tests), the converged FIRE2 density to 1e-8 in max-norm and three
DDFT steps to 1e-10, as in the Python-API driver tests; Picard after 30
iterations to 1e-10, a split-operator step to 1e-11 and a Crank-Nicolson step
to 1e-10; the lattice file equal to the oracle's text.
"""
import os
import subprocess

import numpy as np
import pytest

from tests.parity import Problem, force_err, rel_err, smooth_noise

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "classicaldft_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
SHAPE = (16, 16, 16)
DX = 0.25


def compile_check(out_dir):
    exe = os.path.join(out_dir, "host_api_check")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "host_api_check.cpp"),
           "-L", LIBDIR, "-lcdft_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_host_api_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libcdft_b200.so")):
        pytest.skip("libcdft_b200.so not built")
    exe = compile_check(str(tmp_path))
    assert os.path.getsize(exe) > 0


@pytest.mark.gpu
def test_cpp_host_api_matches_oracle(tmp_path):
    from oracle import algorithms as oalg
    exe = compile_check(str(tmp_path))
    pr = Problem(SHAPE, DX, [1.0], "WhiteBearII", inters=[(0, 0, 1.0, 1.0, 1.8)], kT=1.0)
    rng = np.random.default_rng(1)
    rho = 0.4 * (1.0 + 0.05 * smooth_noise(SHAPE, rng))
    vext = 0.3 * smooth_noise(SHAPE, rng)
    rho.tofile(tmp_path / "rho.bin")
    vext.tofile(tmp_path / "vext.bin")
    run = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    out = dict(line.split("=", 1) for line in run.stdout.split())
    val = {k: float(v) for k, v in out.items() if k not in ("grid_error", "size_error")}
    from oracle import crystal as ocr

    # 1. total
    ref = pr.ref([rho], [0.7], [vext])
    assert rel_err(val["free_energy"], ref.free_energy) <= 1e-12
    assert rel_err(val["grand_potential"], ref.grand_potential) <= 1e-12
    force = np.fromfile(tmp_path / "force.bin")
    assert force_err([force], ref.forces) <= 1e-11
    ref0 = pr.ref([rho], [0.7])
    assert rel_err(val["free_energy_nofield"], ref0.free_energy) <= 1e-12
    assert rel_err(val["grand_potential_nofield"], ref0.grand_potential) <= 1e-12
    assert val["callback_omega"] == val["grand_potential_nofield"]
    assert val["stream_equal"] == 1  # total_stream equals total on each state
    assert val["anchor_dF"] <= 1e-9  # mixed, anchored at rho, 1% off it, against FP64 (4e-10 measured)
    assert rel_err(val["a_vdw"], pr.oweights.mean_field[0]["a_vdw"]) <= 1e-12

    # 2. FIRE2 grand potential
    def ofn(r, mu):
        o = pr.ref([r], [mu])
        return o.free_energy, o.grand_potential, o.forces[0]
    fire = oalg.Fire(dt=0.05, dt_max=0.5, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-10, max_steps=4000)
    o = oalg.Minimizer(fire=fire, param=oalg.Unbounded(1e-18)).grand_potential(pr.omodel.grid, ofn, rho, 1.5)
    assert val["min_converged"] == 1 and o.converged
    assert np.max(np.abs(np.fromfile(tmp_path / "min_rho.bin") - o.densities[0])) <= 1e-8
    assert rel_err(val["min_grand_potential"], o.grand_potential) <= 1e-10

    # 3. DDFT
    def dfn(dens):
        r = pr.ref(dens, [0.0])
        return r.grand_potential, r.forces
    sim = oalg.Simulation(step=oalg.StepConfig(dt=2e-3, dt_max=2e-3, fp_tolerance=1e-10), n_steps=3)
    s = sim.run([rho], pr.omodel.grid, dfn)
    assert np.max(np.abs(np.fromfile(tmp_path / "ddft_rho.bin") - s["densities"][0])) <= 1e-10
    assert rel_err(val["ddft_energy"], s["energies"][-1]) <= 1e-11
    assert val["ddft_time"] == pytest.approx(s["times"][-1], rel=1e-15)
    assert val["mass_final"] == pytest.approx(val["mass_initial"], rel=1e-12)

    # 4. Picard, split-operator and Crank-Nicolson steps, snapshots
    def pfn(mu):
        def f(dens):
            r = pr.ref(dens, [mu])
            return r.grand_potential, r.forces
        return f
    op = oalg.Picard(mixing=0.1, tolerance=1e-14, max_iterations=30).solve([rho], pfn(1.5), DX ** 3)
    assert val["picard_iterations"] == op.iterations == 30
    assert np.max(np.abs(np.fromfile(tmp_path / "picard_rho.bin") - op.densities[0])) <= 1e-10
    assert rel_err(val["picard_omega"], op.grand_potential) <= 1e-11
    grid = pr.omodel.grid
    k2 = oalg.compute_k_squared(grid)
    cfg = oalg.StepConfig(dt=1e-3, fp_tolerance=1e-11)
    so, se, _ = oalg.split_operator_step([rho], grid, k2, oalg.diffusion_propagator(k2, 1.0, 1e-3), dfn, cfg)
    assert np.max(np.abs(np.fromfile(tmp_path / "split_rho.bin") - so[0])) <= 1e-11
    assert rel_err(val["split_energy"], se) <= 1e-11
    co, ce, _ = oalg.crank_nicholson_step([rho], grid, k2, dfn, cfg)
    assert np.max(np.abs(np.fromfile(tmp_path / "cn_rho.bin") - co[0])) <= 1e-10
    assert rel_err(val["cn_energy"], ce) <= 1e-11
    assert val["snapshots"] == 3 and val["snapshot_last_step"] == 4 and val["recorded"] == 1
    s2 = oalg.Simulation(step=oalg.StepConfig(dt=2e-3, dt_max=2e-3, fp_tolerance=1e-10), n_steps=2).run(
        [rho], grid, dfn)
    assert np.max(np.abs(np.fromfile(tmp_path / "snap2_rho.bin") - s2["densities"][0])) <= 1e-10

    # 5. lattice
    pos, dims = ocr.build_lattice(ocr.HCP, ocr.O010, (2, 1, 2))
    assert val["lattice_sites"] == len(pos) and val["lattice_dim_y"] == dims[1]
    assert (tmp_path / "lattice.xyz").read_text() == ocr.export_text(pos, 0)

    # 6. exception mapping
    assert out["grid_error"] == "invalid_argument"
    assert out["size_error"] == "invalid_argument"
