"""The register-resident transform steps of the fused path
(csrc/fft_reg.cuh), built for the host from the same header and checked
against numpy: both orderings of the split transform in both signs (power-of-two lengths
and the 3 x 2^k lengths of the 48- and 96-point grids), the half-output
DFT of the column passes, and the plane R2C / C2R with the half-complex steps on the y-spectrum.  FP32
arithmetic: tolerances are 2e-6 of the transform's max magnitude, as for the
stage-by-stage building blocks.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 2e-6


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("fftreg") / "libfftreg.so")
    subprocess.run(["g++", "-O2", "-std=c++20", "-shared", "-fPIC", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "classicaldft_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "fft_reg_check.cpp"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    dp = ctypes.POINTER(ctypes.c_double)
    L.fr_transform.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
    L.fr_plane_forward.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.fr_plane_inverse.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.fr_dft_half.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp]
    L.fr_plane_forward_units.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    return L


def ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def err(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30)


@pytest.mark.parametrize("N", [2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 256])
def test_split_transform_both_orderings(lib, N):
    A = lib.fr_split_a(N)
    assert A * (N // A) == N and A >= N // A
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    for spectrum_in in (0, 1):
        for inv in (0, 1):
            re, im = x.real.copy(), x.imag.copy()
            lib.fr_transform(N, spectrum_in, inv, ptr(re), ptr(im))
            ref = np.fft.ifft(x) * N if inv else np.fft.fft(x)
            assert err(re + 1j * im, ref) <= TOL, (spectrum_in, inv)


@pytest.mark.parametrize("R", [4, 8, 12, 16])
def test_half_output_dft(lib, R):
    """One decimation-in-frequency step: the even (h = 0) and odd (h = 1)
    outputs of a length-R DFT, as two threads of the column passes split an
    inverse transform's second half."""
    rng = np.random.default_rng(R + 7)
    x = rng.standard_normal(R) + 1j * rng.standard_normal(R)
    for inv in (0, 1):
        ref = np.fft.ifft(x) * R if inv else np.fft.fft(x)
        for h in (0, 1):
            ore, oim = np.zeros(R // 2), np.zeros(R // 2)
            lib.fr_dft_half(R, inv, h, ptr(x.real.copy()), ptr(x.imag.copy()), ptr(ore), ptr(oim))
            assert err(ore + 1j * oim, ref[h::2]) <= TOL, (inv, h)


@pytest.mark.parametrize("ny,nz", [(2, 4), (16, 16), (32, 64), (64, 32), (128, 128), (16, 8), (128, 16),
                                   (8, 256), (4, 2), (48, 48), (96, 96), (48, 128), (96, 16), (16, 96)])
def test_plane_r2c_and_c2r_on_the_y_spectrum(lib, ny, nz):
    rng = np.random.default_rng(ny * 1000 + nz)
    x = rng.standard_normal((ny, nz))
    ld = nz // 2 + 1
    re, im = np.zeros(ny * ld), np.zeros(ny * ld)
    lib.fr_plane_forward(ny, nz, ptr(np.ascontiguousarray(x.reshape(-1))), ptr(re), ptr(im))
    assert err((re + 1j * im).reshape(ny, ld), np.fft.rfft2(x)) <= TOL
    # a non-Hermitian half spectrum: the C2R of its Hermitian projection
    Y = rng.standard_normal((ny, ld)) + 1j * rng.standard_normal((ny, ld))
    out = np.zeros(ny * nz)
    lib.fr_plane_inverse(ny, nz, ptr(np.ascontiguousarray(Y.real.reshape(-1))),
                         ptr(np.ascontiguousarray(Y.imag.reshape(-1))), ptr(out))
    assert err(out.reshape(ny, nz), np.fft.irfft2(Y, s=(ny, nz)) * ny * nz) <= TOL


@pytest.mark.parametrize("ny,nz", [(16, 16), (32, 64), (128, 128), (48, 48), (96, 96), (48, 128), (16, 96)])
def test_plane_forward_mirror_units(lib, ny, nz):
    """The forward plane pass's post-processing per mirror unit (a task and
    the task holding its mirrors, or two self-mirrored tasks) writes every
    output once and equals the element-by-element post-processing."""
    rng = np.random.default_rng(ny * 7 + nz)
    x = rng.standard_normal((ny, nz))
    ld = nz // 2 + 1
    a_re, a_im = np.zeros((ny, ld)), np.zeros((ny, ld))
    lib.fr_plane_forward(ny, nz, ptr(x), ptr(a_re), ptr(a_im))
    b_re, b_im = np.zeros((ny, ld)), np.zeros((ny, ld))
    assert lib.fr_plane_forward_units(ny, nz, ptr(x), ptr(b_re), ptr(b_im)) == 1
    assert np.array_equal(a_re, b_re) and np.array_equal(a_im, b_im)

