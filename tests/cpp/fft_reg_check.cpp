// Host build of the register-resident transform steps
// (classicaldft_b200/csrc/fft_reg.cuh) for the CPU tests: every task of a
// GPU pass runs here in a sequential loop, with the exchange between the two
// halves of a transform done through an explicit array exactly as the
// kernels index their shared-memory buffers.  C linkage for ctypes; double
// on the interface, float inside.
#include <cmath>
#include <vector>

#include "fft_reg.cuh"

using cdft::fft::cpx;
namespace F = cdft::fft;

namespace {

std::vector<cpx> table(int M) {  // exp(-2 pi i n / M), rounded from FP64
  std::vector<cpx> t(M);
  for (int n = 0; n < M; ++n) {
    const double a = -2.0 * 3.14159265358979323846 * n / M;
    t[n] = {(float)std::cos(a), (float)std::sin(a)};
  }
  return t;
}

// One transform of the sequence x[0..N) (element e at x[e * stride]) in
// either ordering; out is natural order, written back in place.
template <int N, bool INV>
void transform(cpx* x, int stride, bool spectrum_in, const cpx* tw) {
  using S = F::Split<N>;
  constexpr int A = S::A, B = S::B;
  std::vector<cpx> ex((size_t)N);  // ex[n2 * A + k1], as the kernels' exchange
  if (!spectrum_in) {
    for (int n2 = 0; n2 < B; ++n2) {
      cpx a[A];
      for (int n1 = 0; n1 < A; ++n1) a[n1] = x[(B * n1 + n2) * stride];
      F::nat_in<N, INV>(a, n2, tw);
      for (int k1 = 0; k1 < A; ++k1) ex[n2 * A + k1] = a[k1];
    }
    for (int k1 = 0; k1 < A; ++k1) {
      cpx b[B];
      for (int n2 = 0; n2 < B; ++n2) b[n2] = ex[n2 * A + k1];
      F::nat_out<N, INV>(b);
      for (int k2 = 0; k2 < B; ++k2) x[(k1 + A * k2) * stride] = b[k2];
    }
  } else {
    for (int k1 = 0; k1 < A; ++k1) {
      cpx b[B];
      for (int k2 = 0; k2 < B; ++k2) b[k2] = x[(k1 + A * k2) * stride];
      F::spec_in<N, INV>(b, k1, tw);
      for (int n2 = 0; n2 < B; ++n2) ex[n2 * A + k1] = b[n2];
    }
    for (int n2 = 0; n2 < B; ++n2) {
      cpx a[A];
      for (int k1 = 0; k1 < A; ++k1) a[k1] = ex[n2 * A + k1];
      F::spec_out<N, INV>(a);
      for (int n1 = 0; n1 < A; ++n1) x[(B * n1 + n2) * stride] = a[n1];
    }
  }
}

template <bool INV>
void transform_rt(int N, cpx* x, int stride, bool spectrum_in, const cpx* tw) {
  switch (N) {
    case 1: break;  // a length-1 transform is the identity
    case 2: transform<2, INV>(x, stride, spectrum_in, tw); break;
    case 4: transform<4, INV>(x, stride, spectrum_in, tw); break;
    case 8: transform<8, INV>(x, stride, spectrum_in, tw); break;
    case 16: transform<16, INV>(x, stride, spectrum_in, tw); break;
    case 32: transform<32, INV>(x, stride, spectrum_in, tw); break;
    case 64: transform<64, INV>(x, stride, spectrum_in, tw); break;
    case 128: transform<128, INV>(x, stride, spectrum_in, tw); break;
    case 3: transform<3, INV>(x, stride, spectrum_in, tw); break;
    case 6: transform<6, INV>(x, stride, spectrum_in, tw); break;
    case 12: transform<12, INV>(x, stride, spectrum_in, tw); break;
    case 24: transform<24, INV>(x, stride, spectrum_in, tw); break;
    case 48: transform<48, INV>(x, stride, spectrum_in, tw); break;
    case 96: transform<96, INV>(x, stride, spectrum_in, tw); break;
    default: transform<256, INV>(x, stride, spectrum_in, tw); break;
  }
}

}  // namespace

extern "C" {

int fr_split_a(int N) { return F::split_a(N); }

// The outputs X[2m + h] of one length-R DFT (decimation in frequency).
void fr_dft_half(int R, int inv, int h, const double* re, const double* im, double* out_re, double* out_im) {
  cpx a[16], o[8];
  for (int i = 0; i < R; ++i) a[i] = {(float)re[i], (float)im[i]};
  auto run = [&](auto rc, auto ic) {
    constexpr int RR = decltype(rc)::value;
    F::dft_half<RR, decltype(ic)::value>(a, h, o);
  };
  using std::integral_constant;
  switch (R * 2 + (inv ? 1 : 0)) {
    case 8: run(integral_constant<int, 4>{}, std::false_type{}); break;
    case 9: run(integral_constant<int, 4>{}, std::true_type{}); break;
    case 16: run(integral_constant<int, 8>{}, std::false_type{}); break;
    case 17: run(integral_constant<int, 8>{}, std::true_type{}); break;
    case 24: run(integral_constant<int, 12>{}, std::false_type{}); break;
    case 25: run(integral_constant<int, 12>{}, std::true_type{}); break;
    case 32: run(integral_constant<int, 16>{}, std::false_type{}); break;
    default: run(integral_constant<int, 16>{}, std::true_type{}); break;
  }
  for (int m = 0; m < R / 2; ++m) {
    out_re[m] = o[m].x;
    out_im[m] = o[m].y;
  }
}

// One complex transform: spectrum_in selects the ordering, inv the sign.
void fr_transform(int N, int spectrum_in, int inv, double* re, double* im) {
  std::vector<cpx> x(N);
  for (int i = 0; i < N; ++i) x[i] = {(float)re[i], (float)im[i]};
  const auto tw = table(N);
  if (inv)
    transform_rt<true>(N, x.data(), 1, spectrum_in != 0, tw.data());
  else
    transform_rt<false>(N, x.data(), 1, spectrum_in != 0, tw.data());
  for (int i = 0; i < N; ++i) {
    re[i] = x[i].x;
    im[i] = x[i].y;
  }
}

// The forward plane pass: z transforms of the pairs x[2n] + i x[2n+1] of
// every row, y transforms of the M packed columns, post-processing on the
// y-spectrum.  real: ny*nz; out: ny*(nz/2+1).
void fr_plane_forward(int ny, int nz, const double* real, double* out_re, double* out_im) {
  const int M = nz / 2, ld = M + 1;
  std::vector<cpx> Z((size_t)ny * M);
  for (int y = 0; y < ny; ++y)
    for (int n = 0; n < M; ++n)
      Z[(size_t)y * M + n] = {(float)real[(size_t)y * nz + 2 * n], (float)real[(size_t)y * nz + 2 * n + 1]};
  const auto twz = table(M), tw2 = table(nz), twy = table(ny);
  for (int y = 0; y < ny; ++y) transform_rt<false>(M, &Z[(size_t)y * M], 1, false, twz.data());
  for (int kz = 0; kz < M; ++kz) transform_rt<false>(ny, &Z[kz], M, false, twy.data());
  for (int ky = 0; ky < ny; ++ky) {
    const int km = (ny - ky) % ny;
    for (int kz = 0; kz < M; ++kz) {
      cpx x0, xM;
      if (kz == 0) {
        F::r2c_post_2d_dc(Z[(size_t)ky * M], Z[(size_t)km * M], x0, xM);
        out_re[(size_t)ky * ld] = x0.x;
        out_im[(size_t)ky * ld] = x0.y;
        out_re[(size_t)ky * ld + M] = xM.x;
        out_im[(size_t)ky * ld + M] = xM.y;
      } else {
        const cpx v = F::r2c_post_2d(Z[(size_t)ky * M + kz], Z[(size_t)km * M + (M - kz)], tw2[kz]);
        out_re[(size_t)ky * ld + kz] = v.x;
        out_im[(size_t)ky * ld + kz] = v.y;
      }
    }
  }
}

// The forward plane pass with the post-processing done per mirror unit
// (F::mirror_unit) from the tasks' y-spectrum columns, as the kernel's
// threads do; every output element written exactly once (count[] checks).
int fr_plane_forward_units(int ny, int nz, const double* real, double* out_re, double* out_im) {
  const int M = nz / 2, ld = M + 1;
  const int AY = F::split_a(ny), BY = ny / AY;
  std::vector<cpx> Z((size_t)ny * M);
  for (int y = 0; y < ny; ++y)
    for (int n = 0; n < M; ++n)
      Z[(size_t)y * M + n] = {(float)real[(size_t)y * nz + 2 * n], (float)real[(size_t)y * nz + 2 * n + 1]};
  const auto twz = table(M), tw2 = table(nz), twy = table(ny);
  for (int y = 0; y < ny; ++y) transform_rt<false>(M, &Z[(size_t)y * M], 1, false, twz.data());
  for (int kz = 0; kz < M; ++kz) transform_rt<false>(ny, &Z[kz], M, false, twy.data());
  std::vector<int> count((size_t)ny * ld, 0);
  auto task = [&](int kz, int k1, std::vector<cpx>& z) {
    z.resize(BY);
    for (int k2 = 0; k2 < BY; ++k2) z[k2] = Z[(size_t)(k1 + AY * k2) * M + kz];
  };
  auto post = [&](const std::vector<cpx>& zt, const std::vector<cpx>& zp, int k1, int kz) {
    for (int k2 = 0; k2 < BY; ++k2) {
      const int ky = k1 + AY * k2;
      const cpx zm = zp[F::mirror_k2(k1, k2, BY)];
      if (kz == 0) {
        cpx x0, xM;
        F::r2c_post_2d_dc(zt[k2], zm, x0, xM);
        out_re[(size_t)ky * ld] = x0.x, out_im[(size_t)ky * ld] = x0.y;
        out_re[(size_t)ky * ld + M] = xM.x, out_im[(size_t)ky * ld + M] = xM.y;
        ++count[(size_t)ky * ld], ++count[(size_t)ky * ld + M];
      } else {
        const cpx v = F::r2c_post_2d(zt[k2], zm, tw2[kz]);
        out_re[(size_t)ky * ld + kz] = v.x, out_im[(size_t)ky * ld + kz] = v.y;
        ++count[(size_t)ky * ld + kz];
      }
    }
  };
  std::vector<cpx> za, zb;
  for (int u = 0; u < M * AY / 2; ++u) {
    const F::MirrorUnit m = F::mirror_unit(u, M, AY);
    task(m.kzA, m.k1A, za);
    task(m.kzB, m.k1B, zb);
    post(za, m.self ? za : zb, m.k1A, m.kzA);
    post(zb, m.self ? zb : za, m.k1B, m.kzB);
  }
  for (int c : count)
    if (c != 1) return 0;
  return 1;
}

// The inverse plane pass (unnormalised C2R of the Hermitian projection):
// pre-processing on the y-spectrum, inverse y transforms of the M packed
// columns, inverse z transforms of the rows, samples doubled.
void fr_plane_inverse(int ny, int nz, const double* in_re, const double* in_im, double* real) {
  const int M = nz / 2, ld = M + 1;
  auto X = [&](int ky, int kz) {
    return cpx{(float)in_re[(size_t)ky * ld + kz], (float)in_im[(size_t)ky * ld + kz]};
  };
  const auto twz = table(M), tw2 = table(nz), twy = table(ny);
  std::vector<cpx> Z((size_t)ny * M);
  for (int ky = 0; ky < ny; ++ky) {
    const int km = (ny - ky) % ny;
    for (int kz = 0; kz < M; ++kz)
      Z[(size_t)ky * M + kz] = kz == 0 ? F::c2r_pre_2d_dc(X(ky, 0), X(km, 0), X(ky, M), X(km, M))
                                       : F::c2r_pre_2d(X(ky, kz), X(km, M - kz), tw2[kz]);
  }
  for (int kz = 0; kz < M; ++kz) transform_rt<true>(ny, &Z[kz], M, true, twy.data());
  for (int y = 0; y < ny; ++y) transform_rt<true>(M, &Z[(size_t)y * M], 1, true, twz.data());
  for (int y = 0; y < ny; ++y)
    for (int n = 0; n < M; ++n) {
      real[(size_t)y * nz + 2 * n] = 2.0 * Z[(size_t)y * M + n].x;
      real[(size_t)y * nz + 2 * n + 1] = 2.0 * Z[(size_t)y * M + n].y;
    }
}

}  // extern "C"
