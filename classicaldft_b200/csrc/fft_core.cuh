// In-place power-of-two FFT building blocks for the fused transform path
// (fft_kernels.cuh): radix-4 stages (one radix-2 stage when log2 M is odd),
// decimation in frequency (natural order in, digit-reversed order out) and in
// time (digit-reversed in, natural out), plus the real<->half-complex
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

#ifdef __CUDACC__
#define CDFT_HD __host__ __device__ __forceinline__
#else
#define CDFT_HD inline
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

CDFT_HD int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

// Radix plan of a length-M transform (M = 2^m): stage s has radix 2 for s = 0
// when m is odd, else 4.  Number of stages and radix of stage s.
CDFT_HD int n_stages(int M) {
  const int m = ilog2(M);
  return (m + 1) / 2;
}
CDFT_HD int stage_radix(int M, int s) {
  const int m = ilog2(M);
  return (s == 0 && (m & 1)) ? 2 : 4;
}

// Sub-transform length of DIF stage s (L_0 = M).
CDFT_HD int dif_length(int M, int s) {
  int L = M;
  for (int q = 0; q < s; ++q) L /= stage_radix(M, q);
  return L;
}

// After all DIF stages, slot p holds X[k] with k = dif_order(M, p): the digits
// of p (most significant first, radices in stage order) become the digits of
// k (least significant first).
CDFT_HD int dif_order(int M, int p) {
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
CDFT_HD int dif_slot(int M, int k) {
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

// Radix-4 DFT in registers with exp(-/+ 2 pi i q t / 4).
template <bool INV>
CDFT_HD void dft4(cpx& a0, cpx& a1, cpx& a2, cpx& a3) {
  const cpx t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = a1 - a3;
  a0 = t0 + t2;
  a2 = t0 - t2;
  a1 = INV ? t1 + mul_i(t3) : t1 + mul_mi(t3);
  a3 = INV ? t1 + mul_mi(t3) : t1 + mul_i(t3);
}

// One DIF butterfly: stage with sub-transform length L and radix r, item w in
// [0, M / r).  Natural order in, dif_order out after the last stage.
template <bool INV>
CDFT_HD void dif_item(cpx* x, int stride, int M, int L, int r, int w, const cpx* tw) {
  const int span = L / r;
  const int j = w % span;
  const int base = (w / span) * L + j;
  if (r == 4) {
    cpx a0 = x[base * stride], a1 = x[(base + span) * stride], a2 = x[(base + 2 * span) * stride],
        a3 = x[(base + 3 * span) * stride];
    dft4<INV>(a0, a1, a2, a3);
    x[base * stride] = a0;
    x[(base + span) * stride] = cmul(a1, twiddle<INV>(tw, M, L, j));
    x[(base + 2 * span) * stride] = cmul(a2, twiddle<INV>(tw, M, L, 2 * j));
    x[(base + 3 * span) * stride] = cmul(a3, twiddle<INV>(tw, M, L, 3 * j));
  } else {
    const cpx a0 = x[base * stride], a1 = x[(base + span) * stride];
    x[base * stride] = a0 + a1;
    x[(base + span) * stride] = cmul(a0 - a1, twiddle<INV>(tw, M, L, j));
  }
}

// One DIT butterfly, the mirror of dif_item.  Stages run in the reverse order
// (the DIF plan's stage 0 last), so dif_order input becomes natural output;
// the inverse DIT after the forward DIF is M times the identity.
template <bool INV>
CDFT_HD void dit_item(cpx* x, int stride, int M, int L, int r, int w, const cpx* tw) {
  const int span = L / r;
  const int j = w % span;
  const int base = (w / span) * L + j;
  if (r == 4) {
    cpx a0 = x[base * stride];
    cpx a1 = cmul(x[(base + span) * stride], twiddle<INV>(tw, M, L, j));
    cpx a2 = cmul(x[(base + 2 * span) * stride], twiddle<INV>(tw, M, L, 2 * j));
    cpx a3 = cmul(x[(base + 3 * span) * stride], twiddle<INV>(tw, M, L, 3 * j));
    dft4<INV>(a0, a1, a2, a3);
    x[base * stride] = a0;
    x[(base + span) * stride] = a1;
    x[(base + 2 * span) * stride] = a2;
    x[(base + 3 * span) * stride] = a3;
  } else {
    const cpx a0 = x[base * stride];
    const cpx a1 = cmul(x[(base + span) * stride], twiddle<INV>(tw, M, L, j));
    x[base * stride] = a0 + a1;
    x[(base + span) * stride] = a0 - a1;
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
