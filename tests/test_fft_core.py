"""The FFT building blocks of the fused transform path (csrc/fft_core.cuh),
built for the host from the same header and checked against numpy: digit
order, DIF / DIT forward and inverse, and the plane R2C / C2R the plane
kernels perform.  FP32 arithmetic: tolerances are 2e-6 of the transform's
max magnitude (cuFFT's single-precision accuracy is of the same order).
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
    out = str(tmp_path_factory.mktemp("fftcore") / "libfftcore.so")
    subprocess.run(["g++", "-O2", "-std=c++20", "-shared", "-fPIC", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "classicaldft_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "fft_core_check.cpp"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    dp = ctypes.POINTER(ctypes.c_double)
    L.fc_transform.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
    L.fc_plane_forward.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.fc_plane_inverse.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    return L


def ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def transform(L, x, dit, inv):
    re = np.ascontiguousarray(x.real, dtype=np.float64)
    im = np.ascontiguousarray(x.imag, dtype=np.float64)
    L.fc_transform(x.size, dit, inv, ptr(re), ptr(im))
    return re + 1j * im


def err(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30)


@pytest.mark.parametrize("M", [2, 4, 8, 16, 32, 64, 128, 256])
def test_digit_order_and_one_dimensional_transforms(lib, M):
    order = np.array([lib.fc_dif_order(M, p) for p in range(M)])
    slot = np.array([lib.fc_dif_slot(M, k) for k in range(M)])
    assert sorted(order) == list(range(M))
    assert np.array_equal(order[slot], np.arange(M))
    rng = np.random.default_rng(M)
    x = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    X = np.fft.fft(x)
    Xi = np.fft.ifft(x) * M
    # DIF: natural in, slot p holds X[order[p]]
    assert err(transform(lib, x, 0, 0), X[order]) <= TOL
    assert err(transform(lib, x, 0, 1), Xi[order]) <= TOL
    # DIT: slot-ordered in, natural out
    assert err(transform(lib, x[order], 1, 0), X) <= TOL
    assert err(transform(lib, x[order], 1, 1), Xi) <= TOL
    # forward DIF then inverse DIT: M x
    assert err(transform(lib, transform(lib, x, 0, 0), 1, 1), M * x) <= TOL


@pytest.mark.parametrize("ny,nz", [(2, 4), (16, 16), (32, 64), (64, 32), (128, 128), (8, 256), (4, 2)])
def test_plane_r2c_and_c2r_match_numpy(lib, ny, nz):
    rng = np.random.default_rng(ny * 1000 + nz)
    x = rng.standard_normal((ny, nz))
    ld = nz // 2 + 1
    re, im = np.zeros(ny * ld), np.zeros(ny * ld)
    lib.fc_plane_forward(ny, nz, ptr(np.ascontiguousarray(x.reshape(-1))), ptr(re), ptr(im))
    X = np.fft.rfft2(x)
    assert err((re + 1j * im).reshape(ny, ld), X) <= TOL
    # inverse of a non-Hermitian half spectrum: numpy's irfft2 is the inverse
    # of its Hermitian projection, as FFTW's and cuFFT's c2r
    Y = rng.standard_normal((ny, ld)) + 1j * rng.standard_normal((ny, ld))
    out = np.zeros(ny * nz)
    lib.fc_plane_inverse(ny, nz, ptr(np.ascontiguousarray(Y.real.reshape(-1))),
                         ptr(np.ascontiguousarray(Y.imag.reshape(-1))), ptr(out))
    ref = np.fft.irfft2(Y, s=(ny, nz)) * ny * nz
    assert err(out.reshape(ny, nz), ref) <= TOL
