// Host build of the FFT building blocks (classicaldft_b200/csrc/fft_core.cuh)
// for the CPU tests: the same item functions the GPU kernels run, driven by
// sequential loops in the order the kernels' stages run.  Exposed with C
// linkage for ctypes; every array is double on the interface and float
// inside, as on the GPU.
#include <cmath>
#include <vector>

#include "fft_core.cuh"

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

template <bool INV>
void dif_all(cpx* x, int stride, int M, const cpx* tw) {
  for (int s = 0; s < F::n_stages(M); ++s) {
    const int r = F::stage_radix(M, s), L = F::dif_length(M, s);
    for (int w = 0; w < M / r; ++w) F::dif_item<INV>(x, stride, M, L, r, w, tw);
  }
}

template <bool INV>
void dit_all(cpx* x, int stride, int M, const cpx* tw) {
  for (int s = F::n_stages(M) - 1; s >= 0; --s) {
    const int r = F::stage_radix(M, s), L = F::dif_length(M, s);
    for (int w = 0; w < M / r; ++w) F::dit_item<INV>(x, stride, M, L, r, w, tw);
  }
}

}  // namespace

extern "C" {

int fc_dif_order(int M, int p) { return F::dif_order(M, p); }
int fc_dif_slot(int M, int k) { return F::dif_slot(M, k); }

// In-place DIF (dit = 0) or DIT (dit = 1) of one complex sequence, forward or inverse.
void fc_transform(int M, int dit, int inv, double* re, double* im) {
  std::vector<cpx> x(M);
  for (int i = 0; i < M; ++i) x[i] = {(float)re[i], (float)im[i]};
  const auto tw = table(M);
  if (!dit && !inv) dif_all<false>(x.data(), 1, M, tw.data());
  if (!dit && inv) dif_all<true>(x.data(), 1, M, tw.data());
  if (dit && !inv) dit_all<false>(x.data(), 1, M, tw.data());
  if (dit && inv) dit_all<true>(x.data(), 1, M, tw.data());
  for (int i = 0; i < M; ++i) {
    re[i] = x[i].x;
    im[i] = x[i].y;
  }
}

// Forward plane transform as the plane kernel does it: R2C along z (pairs
// placed in DIT input order, DIT, post-processing), DIF along y, rows read
// back in natural order.  real: ny*nz; out: ny*(nz/2+1).
void fc_plane_forward(int ny, int nz, const double* real, double* out_re, double* out_im) {
  const int M = nz / 2, ld = M + 1;
  std::vector<cpx> P((size_t)ny * ld);
  for (int iy = 0; iy < ny; ++iy)
    for (int n = 0; n < M; ++n)
      P[(size_t)iy * ld + F::dif_slot(M, n)] = {(float)real[(size_t)iy * nz + 2 * n],
                                                 (float)real[(size_t)iy * nz + 2 * n + 1]};
  const auto twz = table(M), tw2 = table(nz), twy = table(ny);
  for (int iy = 0; iy < ny; ++iy) {
    dit_all<false>(&P[(size_t)iy * ld], 1, M, twz.data());
    for (int k = 0; k <= M / 2; ++k) F::r2c_post_item(&P[(size_t)iy * ld], 1, M, k, tw2.data());
  }
  for (int kz = 0; kz < ld; ++kz) dif_all<false>(&P[kz], ld, ny, twy.data());
  for (int ky = 0; ky < ny; ++ky)
    for (int kz = 0; kz < ld; ++kz) {
      const cpx v = P[(size_t)F::dif_slot(ny, ky) * ld + kz];
      out_re[(size_t)ky * ld + kz] = v.x;
      out_im[(size_t)ky * ld + kz] = v.y;
    }
}

// Inverse plane transform (unnormalised C2R of the Hermitian projection):
// DIF^-1 along y, pre-processing, DIF^-1 along z, read back in natural order.
void fc_plane_inverse(int ny, int nz, const double* in_re, const double* in_im, double* real) {
  const int M = nz / 2, ld = M + 1;
  std::vector<cpx> P((size_t)ny * ld);
  for (int ky = 0; ky < ny; ++ky)
    for (int kz = 0; kz < ld; ++kz)
      P[(size_t)ky * ld + kz] = {(float)in_re[(size_t)ky * ld + kz], (float)in_im[(size_t)ky * ld + kz]};
  const auto twz = table(M), tw2 = table(nz), twy = table(ny);
  for (int kz = 0; kz < ld; ++kz) dif_all<true>(&P[kz], ld, ny, twy.data());
  for (int p = 0; p < ny; ++p) {
    for (int k = 0; k <= M / 2; ++k) F::c2r_pre_item(&P[(size_t)p * ld], 1, M, k, tw2.data());
    dif_all<true>(&P[(size_t)p * ld], 1, M, twz.data());
  }
  for (int iy = 0; iy < ny; ++iy)
    for (int n = 0; n < M; ++n) {
      const cpx v = P[(size_t)F::dif_slot(ny, iy) * ld + F::dif_slot(M, n)];
      real[(size_t)iy * nz + 2 * n] = 2.0 * v.x;
      real[(size_t)iy * nz + 2 * n + 1] = 2.0 * v.y;
    }
}

}  // extern "C"
