// Register-resident building blocks of the fused transform path: a
// power-of-two transform of length N = A * B is two in-register DFTs with
// one exchange between them (the "four-step" split), so a sequence passes
// through shared memory once instead of once per radix stage.
//
//   n = B n1 + n2,  k = k1 + A k2       (n1, k1 < A;  n2, k2 < B)
//   X[k1 + A k2] = sum_n2 w_B^(n2 k2) [ w_N^(n2 k1) sum_n1 x[B n1 + n2] w_A^(n1 k1) ]
//
// Two orderings of the same factorisation:
//   natural-sample input (nat_in, then nat_out): a task (n2) holds the A
//     samples x[B n1 + n2]; after the exchange a task (k1) holds the B
//     spectrum values X[k1 + A k2];
//   natural-spectrum input (spec_in, then spec_out): a task (k1) holds
//     X[k1 + A k2]; after the exchange a task (n2) holds x[B n1 + n2].
// Either ordering runs either sign (INV: exp(+2 pi i n k / N), unnormalised,
// as cuFFT's inverse).  The exchange itself (which task reads which value)
// is the caller's: value k1 of task n2 (nat_in) is value n2 of task k1
// (nat_out), and value n2 of task k1 (spec_in) is value k1 of task n2
// (spec_out).
//
// The half-complex steps of a real 2-D plane transform are done on the
// y-spectrum (before the y inverse, after the y forward), pairing (ky, kz)
// with (-ky, M - kz); see c2r_pre_2d and r2c_post_2d.  Same header on the
// host (g++), where a test drives these steps against numpy.
#pragma once

#include "fft_core.cuh"

namespace cdft {
namespace fft {

// N = A * B with A >= B: powers of two split as evenly as possible; the
// lengths 3 * 2^k of the 48- and 96-point grids into in-register DFTs of at
// most 12 points (3 = 3 x 1, 6 = 3 x 2, 12 = 4 x 3, 24 = 8 x 3, 48 = 8 x 6,
// 96 = 12 x 8).
CDFT_HD constexpr int split_a(int N) {
  if ((N & (N - 1)) == 0) return 1 << ((ilog2(N) + 1) / 2);
  switch (N) {
    case 3: return 3;
    case 6: return 3;
    case 12: return 4;
    case 24: return 8;
    case 48: return 8;
    case 96: return 12;
    default: return 0;
  }
}

template <int N>
struct Split {
  static constexpr int A = split_a(N);
  static constexpr int B = N / A;
  static_assert(A > 0 && A * B == N, "unsupported transform length");
};

// tw[m] = exp(-2 pi i m / N), m < N; the inverse uses its conjugate.
template <bool INV>
CDFT_HD cpx tw_n(const cpx* tw, int m) {
  const cpx w = tw[m];
  return INV ? conj(w) : w;
}

// a[n1] = x[B n1 + n2]  ->  a[k1] = w_N^(n2 k1) sum_n1 x[B n1 + n2] w_A^(n1 k1)
template <int N, bool INV>
CDFT_HD void nat_in(cpx* a, int n2, const cpx* tw) {
  constexpr int A = Split<N>::A;
  dft<A, INV>(a);
  if (n2 != 0) {
CDFT_UNROLL
    for (int k1 = 1; k1 < A; ++k1) a[k1] = cmul(a[k1], tw_n<INV>(tw, n2 * k1));
  }
}

// b[n2] (value k1 of every task n2)  ->  b[k2] = X[k1 + A k2]
template <int N, bool INV>
CDFT_HD void nat_out(cpx* b) {
  dft<Split<N>::B, INV>(b);
}

// b[k2] = X[k1 + A k2]  ->  b[n2] = w_N^(n2 k1) sum_k2 X[k1 + A k2] w_B^(n2 k2)
template <int N, bool INV>
CDFT_HD void spec_in(cpx* b, int k1, const cpx* tw) {
  constexpr int B = Split<N>::B;
  dft<B, INV>(b);
  if (k1 != 0) {
CDFT_UNROLL
    for (int n2 = 1; n2 < B; ++n2) b[n2] = cmul(b[n2], tw_n<INV>(tw, n2 * k1));
  }
}

// a[k1] (value n2 of every task k1)  ->  a[n1] = x[B n1 + n2]
template <int N, bool INV>
CDFT_HD void spec_out(cpx* a) {
  dft<Split<N>::A, INV>(a);
}

// Half-complex-to-real pre-processing of a plane on its y-spectrum.  The
// plane X[ky][kz] (kz = 0..M) is the spectrum of a real NY x 2M array; the
// result Zk[ky][kz] (kz < M) is such that the inverse y transform of Zk and
// then the inverse length-M z transform of each row give M (x[y][2n] + i
// x[y][2n+1]) / 2 (the caller doubles): the length-2M C2R of each row done
// as a length-M complex transform, moved onto the y-spectrum (the conjugate
// of a row value at kz is the y-spectrum value at (-ky, kz), conjugated).
// xm is X at the mirror (-ky mod NY, M - kz) for kz in 1..M-1.  For kz = 0, x0m and xM, xMm are X[-ky][0], X[ky][M],
// X[-ky][M]: only the real parts of the rows' kz = 0 and M values enter
// (the C2R of the Hermitian projection), and a real part is (X + conj
// X_mirror) / 2 on the spectrum.
CDFT_HD cpx c2r_pre_2d(cpx xk, cpx xm, cpx tw2k) {
  const cpx e = scale(xk + conj(xm), 0.5f);
  const cpx o = cmul(scale(xk - conj(xm), 0.5f), conj(tw2k));
  return e + mul_i(o);
}
CDFT_HD cpx c2r_pre_2d_dc(cpx x0, cpx x0m, cpx xM, cpx xMm) {
  const cpx p0 = scale(x0 + conj(x0m), 0.5f);
  const cpx pm = scale(xM + conj(xMm), 0.5f);
  return scale(p0 + pm, 0.5f) + mul_i(scale(p0 - pm, 0.5f));
}

// Mirror-pair units of a forward plane pass's y-spectrum tasks (kz, k1),
// kz < M, k1 < AY, each task holding Z[k1 + AY k2][kz] for k2 < BY.  The
// post-processing of element (ky, kz) needs its mirror (-ky, M - kz mod M),
// which lies in task ((M - kz) mod M, (AY - k1) mod AY).  Unit u < M AY / 2
// is a task A and the task B holding the mirrors of A's elements (and A
// those of B's), or, for the four self-mirrored tasks (kz in {0, M/2}, k1
// in {0, AY/2}), two of them side by side (self = true), so one thread
// finishes a unit without an exchange.  M and AY even.
struct MirrorUnit {
  int kzA, k1A, kzB, k1B;
  bool self;
};
CDFT_HD MirrorUnit mirror_unit(int u, int M, int AY) {
  const int half = M / 2, c = u % half, r = u / half;
  MirrorUnit m;
  if (c != 0) {
    m.kzA = c, m.k1A = r, m.kzB = M - c, m.k1B = (AY - r) % AY, m.self = false;
  } else {
    const int kz = r < AY / 2 ? 0 : half, rr = r < AY / 2 ? r : r - AY / 2;
    m.kzA = kz, m.kzB = kz, m.k1A = rr, m.self = rr == 0;
    m.k1B = rr == 0 ? AY / 2 : AY - rr;
  }
  return m;
}
// Index, in the task holding it, of the mirror of element k2 of a task k1.
CDFT_HD int mirror_k2(int k1, int k2, int BY) { return k1 == 0 ? (BY - k2) % BY : BY - 1 - k2; }

// Real-to-half-complex post-processing on the y-spectrum: Z[ky][kz] (kz <
// M) is the forward y transform of the rows' forward length-M transforms of
// z[n] = x[2n] + i x[2n+1]; X[ky][kz] for kz in 1..M-1 from Z[ky][kz] and
// zm = Z[-ky][M - kz]: X[k] = E + w^k O with E = (Z[k] + conj Z[M-k]) / 2,
// O = -i (Z[k] - conj Z[M-k]) / 2 per row, moved onto the y-spectrum.  kz =
// 0 gives X[ky][0] = E + O and X[ky][M] = E - O from Z[ky][0] and Z[-ky][0].
CDFT_HD cpx r2c_post_2d(cpx zk, cpx zm, cpx tw2k) {
  const cpx e = scale(zk + conj(zm), 0.5f);
  const cpx o = scale(mul_mi(zk - conj(zm)), 0.5f);
  return e + cmul(o, tw2k);
}
CDFT_HD void r2c_post_2d_dc(cpx z0, cpx z0m, cpx& x0, cpx& xM) {
  const cpx e = scale(z0 + conj(z0m), 0.5f);
  const cpx o = scale(mul_mi(z0 - conj(z0m)), 0.5f);
  x0 = e + o;
  xM = e - o;
}

}  // namespace fft
}  // namespace cdft
