// In-place power-of-two FFT building blocks for the fused transform path
// (fft_kernels.cuh): radix-16 stages, then one radix-8, -4 or -2 stage for
// the rest (128 = 16 x 8, 64 = 16 x 4, 32 = 16 x 2), each butterfly an
// in-register DFT; decimation in frequency (natural order in, digit-reversed
// order out) and in time (digit-reversed in, natural out), plus the real<->half-complex
// pre/post-processing of a length-2M real transform done as a length-M
// complex one.  Conventions are cuFFT's (and FFTW's): forward exp(-2 pi i
// n k / M), inverse exp(+2 pi i n k / M), no normalisation.
//
// Every function works on one butterfly (or one pair) of one sequence whose
// element e lives at x[e * stride]; a kernel runs all items of a stage across
// its threads and synchronises between stages.  The same header compiles for
// the host (g++), where a test program checks the index algebra and the
// arithmetic against numpy.
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

// Radix plan of a length-M transform (M = 2^m): radix 16 for the first
// m / 4 stages, then 2^(m mod 4) for a last stage when m mod 4 != 0.
CDFT_HD constexpr int n_stages(int M) {
  const int m = ilog2(M);
  return m / 4 + ((m % 4) ? 1 : 0);
}
CDFT_HD constexpr int stage_radix(int M, int s) {
  const int m = ilog2(M);
  return (s < m / 4) ? 16 : (1 << (m % 4));
}

// Sub-transform length of DIF stage s (L_0 = M).
CDFT_HD constexpr int dif_length(int M, int s) {
  int L = M;
  for (int q = 0; q < s; ++q) L /= stage_radix(M, q);
  return L;
}

// After all DIF stages, slot p holds X[k] with k = dif_order(M, p): the digits
// of p (most significant first, radices in stage order) become the digits of
// k (least significant first).
CDFT_HD constexpr int dif_order(int M, int p) {
  int k = 0, mult = 1, L = M;
  const int ns = n_stages(M);
  for (int s = 0; s < ns; ++s) {
    const int r = stage_radix(M, s);
    const int Ls = L / r;
    const int d = p / Ls;
    p -= d * Ls;
    k += d * mult;
    mult *= r;
    L = Ls;
  }
  return k;
}

// Inverse of dif_order: the slot that holds frequency (or, for DIT input,
// sample) k.
CDFT_HD constexpr int dif_slot(int M, int k) {
  int p = 0, L = M;
  const int ns = n_stages(M);
  for (int s = 0; s < ns; ++s) {
    const int r = stage_radix(M, s);
    const int d = k % r;
    k /= r;
    L /= r;
    p += d * L;
  }
  return p;
}

// Twiddle W_L^e from the table tw[n] = exp(-2 pi i n / M) (L divides M).
template <bool INV>
CDFT_HD cpx twiddle(const cpx* tw, int M, int L, int e) {
  const cpx w = tw[(e * (M / L)) & (M - 1)];
  return INV ? conj(w) : w;
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

// One DIF butterfly: stage with sub-transform length L and radix R, item w in
// [0, M / R).  Natural order in, dif_order out after the last stage.
template <int R, bool INV>
CDFT_HD void dif_item_r(cpx* x, int stride, int M, int L, int w, const cpx* tw) {
  const int span = L / R;
  const int j = w % span;
  const int base = (w / span) * L + j;
  cpx a[R];
CDFT_UNROLL
  for (int q = 0; q < R; ++q) a[q] = x[(base + q * span) * stride];
  dft<R, INV>(a);
  x[base * stride] = a[0];
CDFT_UNROLL
  for (int t = 1; t < R; ++t)  // the last stage (L == R) has j = 0: no twiddle
    x[(base + t * span) * stride] = (L == R) ? a[t] : cmul(a[t], twiddle<INV>(tw, M, L, j * t));
}

// One DIT butterfly, the mirror of dif_item_r.  Stages run in the reverse
// order (the DIF plan's stage 0 last), so dif_order input becomes natural
// output; the inverse DIT after the forward DIF is M times the identity.
template <int R, bool INV>
CDFT_HD void dit_item_r(cpx* x, int stride, int M, int L, int w, const cpx* tw) {
  const int span = L / R;
  const int j = w % span;
  const int base = (w / span) * L + j;
  cpx a[R];
  a[0] = x[base * stride];
CDFT_UNROLL
  for (int q = 1; q < R; ++q)  // the first DIT stage (L == R) has j = 0: no twiddle
    a[q] = (L == R) ? x[(base + q * span) * stride] : cmul(x[(base + q * span) * stride], twiddle<INV>(tw, M, L, j * q));
  dft<R, INV>(a);
CDFT_UNROLL
  for (int t = 0; t < R; ++t) x[(base + t * span) * stride] = a[t];
}

// Runtime-radix forms (the host test drives every stage through these).
template <bool INV>
inline void dif_item(cpx* x, int stride, int M, int L, int r, int w, const cpx* tw) {
  switch (r) {
    case 16: dif_item_r<16, INV>(x, stride, M, L, w, tw); break;
    case 8: dif_item_r<8, INV>(x, stride, M, L, w, tw); break;
    case 4: dif_item_r<4, INV>(x, stride, M, L, w, tw); break;
    default: dif_item_r<2, INV>(x, stride, M, L, w, tw); break;
  }
}
template <bool INV>
inline void dit_item(cpx* x, int stride, int M, int L, int r, int w, const cpx* tw) {
  switch (r) {
    case 16: dit_item_r<16, INV>(x, stride, M, L, w, tw); break;
    case 8: dit_item_r<8, INV>(x, stride, M, L, w, tw); break;
    case 4: dit_item_r<4, INV>(x, stride, M, L, w, tw); break;
    default: dit_item_r<2, INV>(x, stride, M, L, w, tw); break;
  }
}

// Real-to-half-complex post-processing of a length-2M real sequence whose
// pairs were transformed as z[n] = x[2n] + i x[2n+1] (Z natural in slots
// 0..M-1).  Pair item k in [0, M/2]: writes X[k] and X[M-k] into slots k and
// M-k (X[M] into slot M, which the caller provides).  tw2[n] = exp(-2 pi i n
// / (2M)).
CDFT_HD void r2c_post_item(cpx* x, int stride, int M, int k, const cpx* tw2) {
  if (k == 0) {
    const cpx z = x[0];
    x[0] = {z.x + z.y, 0.0f};
    x[M * stride] = {z.x - z.y, 0.0f};
    return;
  }
  const int kc = M - k;
  const cpx zk = x[k * stride], zc = x[kc * stride];
  // X[k] = E + W^k O, E = (Z[k] + conj Z[M-k]) / 2, O = -i (Z[k] - conj Z[M-k]) / 2
  const cpx e = scale(zk + conj(zc), 0.5f);
  const cpx o = scale(mul_mi(zk - conj(zc)), 0.5f);
  const cpx xk = e + cmul(o, tw2[k]);
  if (kc == k) {
    x[k * stride] = xk;
    return;
  }
  const cpx xkc = conj(e) + cmul(conj(o), tw2[kc]);  // E[M-k] = conj E[k], O[M-k] = conj O[k]
  x[k * stride] = xk;
  x[kc * stride] = xkc;
}

// Half-complex-to-real pre-processing (the inverse of r2c_post_item): from
// X[0..M] (natural, slots 0..M) to Z[0..M-1] in slots 0..M-1.  The inverse
// length-M transform of Z is M (x[2n] + i x[2n+1]) / 2 for the unnormalised
// length-2M C2R output x, so the caller doubles it on output.  The imaginary
// parts of X[0] and X[M] are dropped (the C2R of the Hermitian projection).
CDFT_HD void c2r_pre_item(cpx* x, int stride, int M, int k, const cpx* tw2) {
  if (k == 0) {
    const float x0 = x[0].x, xm = x[M * stride].x;
    x[0] = {0.5f * (x0 + xm), 0.5f * (x0 - xm)};  // E + i O with E, O real
    return;
  }
  const int kc = M - k;
  const cpx xk = x[k * stride], xc = x[kc * stride];
  // E = (X[k] + conj X[M-k]) / 2,  O = (X[k] - conj X[M-k]) / 2 W^-k,  Z = E + i O
  const cpx e = scale(xk + conj(xc), 0.5f);
  const cpx o = cmul(scale(xk - conj(xc), 0.5f), conj(tw2[k]));
  const cpx zk = e + mul_i(o);
  if (kc == k) {
    x[k * stride] = zk;
    return;
  }
  const cpx e2 = scale(xc + conj(xk), 0.5f);
  const cpx o2 = cmul(scale(xc - conj(xk), 0.5f), conj(tw2[kc]));
  x[k * stride] = zk;
  x[kc * stride] = e2 + mul_i(o2);
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
