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

// On sm_100 a complex sum, difference or real scaling is one packed FP32
// instruction (add / sub / mul .rn.f32x2: both lanes round exactly as the
// scalar instructions do); elsewhere two scalar ones.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
#define CDFT_F32X2 1
__device__ __forceinline__ unsigned long long pack2(cpx a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ cpx unpack2(unsigned long long r) {
  cpx a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
#endif

CDFT_HD cpx operator+(cpx a, cpx b) {
#ifdef CDFT_F32X2
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
  return unpack2(r);
#else
  return {a.x + b.x, a.y + b.y};
#endif
}
CDFT_HD cpx operator-(cpx a, cpx b) {
#ifdef CDFT_F32X2
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
  return unpack2(r);
#else
  return {a.x - b.x, a.y - b.y};
#endif
}
CDFT_HD cpx cmul(cpx a, cpx b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
CDFT_HD cpx conj(cpx a) { return {a.x, -a.y}; }
CDFT_HD cpx mul_i(cpx a) { return {-a.y, a.x}; }   // i a
CDFT_HD cpx mul_mi(cpx a) { return {a.y, -a.x}; }  // -i a
CDFT_HD cpx scale(cpx a, float s) {
#ifdef CDFT_F32X2
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(cpx{s, s})));
  return unpack2(r);
#else
  return {a.x * s, a.y * s};
#endif
}

CDFT_HD constexpr int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

// exp(-/+ 2 pi i t / R) for R dividing 48 (the radices 2, 3, 4, 6, 8, 12,
// 16), as constants: cos(2 pi t / 48) from its first quadrant, cos(k 7.5
// degrees) for k = 0 .. 12 rounded to FP32.
CDFT_HD constexpr float c48(int t) {
  constexpr float q[13] = {1.0f,
                           0.99144486137381038f,
                           0.96592582628906829f,
                           0.92387953251128674f,
                           0.86602540378443865f,
                           0.79335334029123517f,
                           0.70710678118654752f,
                           0.60876142900872066f,
                           0.5f,
                           0.38268343236508977f,
                           0.25881904510252076f,
                           0.13052619222005159f,
                           0.0f};
  t = ((t % 48) + 48) % 48;
  if (t <= 12) return q[t];
  if (t <= 24) return -q[24 - t];
  if (t <= 36) return -q[t - 24];
  return q[48 - t];
}
CDFT_HD constexpr float s48(int t) { return c48(t + 36); }  // sin(x) = cos(x - pi/2)

// a * exp(-/+ 2 pi i t / R), exact for the trivial angles.
template <int R, int T, bool INV>
CDFT_HD cpx rot(cpx a) {
  static_assert(48 % R == 0, "rotation radix must divide 48");
  constexpr int t48 = (T * (48 / R)) % 48;
  if constexpr (t48 == 0) {
    return a;
  } else if constexpr (t48 == 12) {
    return INV ? mul_i(a) : mul_mi(a);
  } else if constexpr (t48 == 24) {
    return {-a.x, -a.y};
  } else if constexpr (t48 == 36) {
    return INV ? mul_mi(a) : mul_i(a);
  } else {
    constexpr float c = c48(t48), sn = INV ? s48(t48) : -s48(t48);
    return {a.x * c - a.y * sn, a.x * sn + a.y * c};
  }
}

// In-register DFT of a[0..R), natural order in and out, R in {1, 2, 3, 4,
// 6, 8, 12, 16}: radix-2 decimation in time recursively down to 2 or 3
// points; the 3-point DFT is X0 = a0 + s, X1,2 = a0 - s/2 -/+ i (sqrt 3 / 2)
// (a1 - a2) with s = a1 + a2 (signs swapped for the inverse).
template <int R, bool INV>
CDFT_HD void dft(cpx* a) {
  if constexpr (R == 2) {
    const cpx t = a[0];
    a[0] = t + a[1];
    a[1] = t - a[1];
  } else if constexpr (R == 3) {
    constexpr float h = 0.86602540378443865f;
    const cpx sum = a[1] + a[2];
    const cpx d = scale(a[1] - a[2], h);
    const cpx m = a[0] - scale(sum, 0.5f);
    a[0] = a[0] + sum;
    a[1] = INV ? m + mul_i(d) : m + mul_mi(d);
    a[2] = INV ? m + mul_mi(d) : m + mul_i(d);
  } else if constexpr (R > 3) {
    static_assert(R % 2 == 0, "DFT length must be 3 times a power of two or a power of two");
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

// Half of the outputs of a length-R DFT by one decimation-in-frequency
// step: out[m] = X[2m + h] for m < R/2 is the length-R/2 DFT of
// (a[k] + (-1)^h a[k + R/2]) w_R^(k h).
template <int R, bool INV>
CDFT_HD void dft_half(const cpx* a, int h, cpx* out) {
  static_assert(R % 2 == 0, "even DFT lengths only");
  if (h == 0) {
CDFT_UNROLL
    for (int k = 0; k < R / 2; ++k) out[k] = a[k] + a[k + R / 2];
  } else {
    [&]<int... T>(std::integer_sequence<int, T...>) {
      ((out[T] = rot<R, T, INV>(a[T] - a[T + R / 2])), ...);
    }(std::make_integer_sequence<int, R / 2>{});
  }
  dft<R / 2, INV>(out);
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
