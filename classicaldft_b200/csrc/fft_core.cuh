// Complex FP32 arithmetic and the in-register DFTs (lengths 2 to 16) the
// fused transform path builds its transforms from (fft_reg.cuh).
// Conventions are cuFFT's (and FFTW's): forward exp(-2 pi i n k / M),
// inverse exp(+2 pi i n k / M), no normalisation.  The same header compiles
// for the host (g++), where a test program checks the arithmetic against
// numpy.
#pragma once

#include <utility>

#ifdef __CUDACC__
#define CDFT_HD __host__ __device__ __forceinline__
#define CDFT_UNROLL _Pragma("unroll")
#else
#define CDFT_HD inline
#define CDFT_UNROLL
#endif

namespace cdft {
namespace fft {

struct alignas(8) cpx {
  float x, y;
};

CDFT_HD cpx operator+(cpx a, cpx b) { return {a.x + b.x, a.y + b.y}; }
CDFT_HD cpx operator-(cpx a, cpx b) { return {a.x - b.x, a.y - b.y}; }
CDFT_HD cpx cmul(cpx a, cpx b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
CDFT_HD cpx conj(cpx a) { return {a.x, -a.y}; }
CDFT_HD cpx mul_i(cpx a) { return {-a.y, a.x}; }   // i a
CDFT_HD cpx mul_mi(cpx a) { return {a.y, -a.x}; }  // -i a
CDFT_HD cpx scale(cpx a, float s) { return {a.x * s, a.y * s}; }

CDFT_HD constexpr int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

// exp(-/+ 2 pi i t / R) for R dividing 16, as constants: cos and sin of
// 2 pi t / 16 for t = 0 .. 15.
CDFT_HD constexpr float c16(int t) {
  constexpr float c[16] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
                           0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f,
                           -1.0f, -0.92387953251128674f, -0.70710678118654752f, -0.38268343236508977f,
                           0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f};
  return c[t & 15];
}
CDFT_HD constexpr float s16(int t) { return c16(t + 12); }  // sin(x) = cos(x - pi/2)

// a * exp(-/+ 2 pi i t / R), exact for the trivial angles.
template <int R, int T, bool INV>
CDFT_HD cpx rot(cpx a) {
  constexpr int t16 = (T * (16 / R)) & 15;
  if constexpr (t16 == 0) {
    return a;
  } else if constexpr (t16 == 4) {
    return INV ? mul_i(a) : mul_mi(a);
  } else if constexpr (t16 == 8) {
    return {-a.x, -a.y};
  } else if constexpr (t16 == 12) {
    return INV ? mul_mi(a) : mul_i(a);
  } else {
    constexpr float c = c16(t16), sn = INV ? s16(t16) : -s16(t16);
    return {a.x * c - a.y * sn, a.x * sn + a.y * c};
  }
}

// In-register DFT of a[0..R), natural order in and out (radix-2 decimation
// in time, recursively), R in {1, 2, 4, 8, 16}.
template <int R, bool INV>
CDFT_HD void dft(cpx* a) {
  if constexpr (R == 2) {
    const cpx t = a[0];
    a[0] = t + a[1];
    a[1] = t - a[1];
  } else if constexpr (R > 2) {
    cpx e[R / 2], o[R / 2];
CDFT_UNROLL
    for (int i = 0; i < R / 2; ++i) {
      e[i] = a[2 * i];
      o[i] = a[2 * i + 1];
    }
    dft<R / 2, INV>(e);
    dft<R / 2, INV>(o);
    [&]<int... T>(std::integer_sequence<int, T...>) {
      ((a[T] = e[T] + rot<R, T, INV>(o[T]), a[T + R / 2] = e[T] - rot<R, T, INV>(o[T])), ...);
    }(std::make_integer_sequence<int, R / 2>{});
  }
}

}  // namespace fft

// Twiddle tables (exp(-2 pi i n / M), FP64-rounded to FP32) of the four
// lengths the fused path uses, back to back in one device array.
struct FftTables {
  const fft::cpx* tx;  // nx entries
  const fft::cpx* ty;  // ny entries
  const fft::cpx* tz;  // nz / 2 entries
  const fft::cpx* t2;  // nz entries (R2C / C2R post- and pre-processing)
};

}  // namespace cdft
