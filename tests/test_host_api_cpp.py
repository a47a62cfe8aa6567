"""The C++ host API (include/dft_b200/dft_b200.hpp): the check program in
tests/cpp is compiled with g++ against the header and libcdft_b200.so (CPU
test), then run on the GPU and compared with the oracle: F and Omega to
1e-12 relative and forces to 1e-11 of their max (the tolerances of the other
FP64 parity tests), the converged FIRE2 density to 1e-8 in max-norm and three
DDFT steps to 1e-10, as in the Python-API driver tests.
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

    # 4. exception mapping
    assert out["grid_error"] == "invalid_argument"
    assert out["size_error"] == "invalid_argument"
