// Pointwise FMT free-energy density Phi(n_alpha) and its partial derivatives,
// for all five models of include/dft/functionals/fmt/models.hpp.
//
// Everything is templated on the scalar type T: T = double gives the primal
// evaluation of the reference (models.hpp:49-81); T = Dual carries a tangent
// through the same arithmetic, which turns the hand-written adjoint dPhi into
// its directional derivative (forward-over-reverse Hessian-vector product).
//
// The f-function derivatives are closed forms of the exact expressions the
// reference differentiates with autodiff (models.hpp:59-61), including the
// eta < 1e-6 Taylor branches (models.hpp:200, 250, 282, 290).
#pragma once

#include "cdft_common.cuh"

namespace cdft {

// ---------------------------------------------------------------- duals

struct Dual {
  double v, d;
};
__host__ __device__ inline Dual mk(double v, double d = 0.0) { return Dual{v, d}; }
__host__ __device__ inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__host__ __device__ inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__host__ __device__ inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
__host__ __device__ inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__host__ __device__ inline Dual operator/(Dual a, Dual b) {
  double q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
__host__ __device__ inline Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__host__ __device__ inline Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__host__ __device__ inline Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__host__ __device__ inline Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__host__ __device__ inline Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__host__ __device__ inline Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__host__ __device__ inline Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__host__ __device__ inline Dual operator/(double a, Dual b) {
  double q = a / b.v;
  return {q, -q * b.d / b.v};
}
__host__ __device__ inline Dual dlog(Dual a) { return {log(a.v), a.d / a.v}; }
__host__ __device__ inline double dlog(double a) { return log(a); }
__host__ __device__ inline double val(double a) { return a; }
__host__ __device__ inline double val(Dual a) { return a.v; }
__host__ __device__ inline double zero_like(double) { return 0.0; }
__host__ __device__ inline Dual zero_like(Dual) { return Dual{0.0, 0.0}; }
template <class T> __host__ __device__ inline T cst(double c) { return T(c); }
template <> __host__ __device__ inline Dual cst<Dual>(double c) { return Dual{c, 0.0}; }

// ------------------------------------------------------------- measures

// Symmetric tensor stored as xx, xy, xz, yy, yz, zz (tensor_index order).
template <class T>
struct Measures {
  T eta, n0, n1, n2;
  T v0[3], v1[3];
  T t[6];
};

template <class T>
struct MeasureDerivs {
  T d_eta, d_n0, d_n1, d_n2;
  T d_v0[3], d_v1[3];
  T d_t[6];  // dPhi/dT_ij for i <= j (the matrix is symmetric)
};

template <class T>
struct FVals {
  T f1, df1, f2, df2, f3, df3;
};

// f1, f2, f3 and their eta-derivatives for one model (models.hpp:153-324).
// log(1 - eta), 1/(1 - eta) and 1/eta are formed once; every other quotient
// of the reference's expressions is rewritten with these reciprocals, which
// keeps the FP64 division count at two per point.
// FAST: the caller guarantees eta >= 1e-6 (no Taylor branch), and the two
// reciprocals come from one: 1/(eta e) times e or eta.
template <int MODEL, class T, bool FAST = false>
__host__ __device__ __forceinline__ FVals<T> fmt_f(T eta) {
  constexpr int model = MODEL;
  constexpr bool needs_ih = model != kRosenfeld && model != kEsFMT;
  FVals<T> r;
  const double ev = val(eta);
  const T e = 1.0 - eta;
  T ie, ih = cst<T>(0.0), ih2 = cst<T>(0.0);
  const bool taylor = FAST ? false : ev < 1e-6;
  if constexpr (FAST && needs_ih) {
    const T rr = 1.0 / (eta * e);
    ie = eta * rr;
    ih = e * rr;
    ih2 = ih * ih;
  } else {
    ie = 1.0 / e;
    if (!taylor && needs_ih) {  // 1/eta only where it is used
      ih = 1.0 / eta;
      ih2 = ih * ih;
    }
  }
  const T ie2 = ie * ie;
  const T lg = dlog(e);
  r.f1 = lg;
  r.df1 = -ie;
  if constexpr (model == kWhiteBearII) {
    if (taylor) {
      r.f2 = 1.0 + eta * (1.0 + eta * (10.0 / 9.0 + (7.0 / 6.0) * eta));
      r.df2 = 1.0 + eta * (2.0 * (10.0 / 9.0) + 3.0 * (7.0 / 6.0) * eta);
    } else {
      r.f2 = (1.0 / 3.0) + (4.0 / 3.0) * ie + (2.0 / 3.0) * ih * lg;
      r.df2 = (4.0 / 3.0) * ie2 - (2.0 / 3.0) * ih2 * lg - (2.0 / 3.0) * ih * ie;
    }
  } else {
    r.f2 = ie;
    r.df2 = ie2;
  }
  if constexpr (model == kRosenfeld || model == kEsFMT) {
    r.f3 = ie2;
    r.df3 = 2.0 * ie2 * ie;
  } else if constexpr (model == kRSLT || model == kWhiteBearI) {
    if (taylor) {
      if constexpr (model == kRSLT) {
        r.f3 = 1.0 + (2.0 / 3.0) * eta + 0.5 * eta * eta;
        r.df3 = (2.0 / 3.0) + eta;
      } else {
        r.f3 = 1.5 + eta * (8.0 / 3.0 + eta * (15.0 / 4.0 + (24.0 / 5.0) * eta));
        r.df3 = 8.0 / 3.0 + eta * (2.0 * (15.0 / 4.0) + 3.0 * (24.0 / 5.0) * eta);
      }
    } else {
      // f3 = 1/(eta e^2) + log(e)/eta^2
      r.f3 = ih * ie2 + lg * ih2;
      r.df3 = -(e - 2.0 * eta) * ih2 * ie2 * ie - ie * ih2 - 2.0 * lg * ih2 * ih;
    }
  } else {  // WhiteBearII
    if (taylor) {
      r.f3 = 1.5 + (7.0 / 3.0) * eta + 3.25 * eta * eta + 4.2 * eta * eta * eta;
      r.df3 = 7.0 / 3.0 + 6.5 * eta + 12.6 * eta * eta;
    } else {
      // f3 = -(1 - 3 eta + eta^2)/(eta e^2) - log(e)/eta^2
      const T g = 1.0 - 3.0 * eta + eta * eta;
      const T gp = -3.0 + 2.0 * eta;
      r.f3 = -(g * ih * ie2) - lg * ih2;
      r.df3 = -(gp * ih * ie2) + g * (e - 2.0 * eta) * ih2 * ie2 * ie + ie * ih2 + 2.0 * lg * ih2 * ih;
    }
  }
  return r;
}

// Phi and all partial derivatives at one point (models.hpp:22-81, 169-357).
// Returns false (and leaves outputs untouched) where eta < 1e-30: the
// reference skips those points (hard_sphere.hpp:199-200).
// ONE: a single species of radius R, for which n0 = a0 n2, n1 = a1 n2 and
// v0 = a1 v1 (a0 = 1/(4 pi R^2), a1 = 1/(4 pi R), hard_sphere.hpp:80-85);
// m.n0, m.n1 and m.v0 are not read, and d_n2 and d_v1 come out with those
// chains folded in (d_n0, d_n1, d_v0 zero):
//   Phi = -a0 n2 f1 + a1 (n2^2 - v1.v1) f2 + Phi3 f3,
//   d_n2 = -a0 f1 + 2 a1 n2 f2 + dPhi3/dn2 f3,  d_v1 = -2 a1 f2 v1 + dPhi3/dv1 f3.
// FAST: the caller guarantees eta >= 1e-6 (see fmt_f); always returns true.
template <int MODEL, class T, bool ONE = false, bool FAST = false>
__host__ __device__ __forceinline__ bool fmt_phi_dphi(double A, double B, const Measures<T>& m, T& phi,
                                                      MeasureDerivs<T>& dm, double a0 = 0.0, double a1 = 0.0) {
  constexpr int model = MODEL;
  constexpr bool tensor = model_has_tensor(MODEL);
  if (!FAST && val(m.eta) < 1e-30) return false;
  constexpr double INV_24PI = 1.0 / (24.0 * kPi);
  constexpr double INV_8PI = 1.0 / (8.0 * kPi);
  constexpr double INV_4PI = 1.0 / (4.0 * kPi);
  constexpr double INV_36PI = 1.0 / (36.0 * kPi);

  // inner products (measures.hpp:34-44); T symmetric
  const T txx = m.t[0], txy = m.t[1], txz = m.t[2], tyy = m.t[3], tyz = m.t[4], tzz = m.t[5];
  T dot01 = zero_like(m.eta);
  if constexpr (!ONE) dot01 = m.v0[0] * m.v1[0] + m.v0[1] * m.v1[1] + m.v0[2] * m.v1[2];
  T dot11 = m.v1[0] * m.v1[0] + m.v1[1] * m.v1[1] + m.v1[2] * m.v1[2];
  T tt[6];   // TT = T*T (symmetric)
  T tv[3];   // T v1
  T trT2 = zero_like(m.eta), trT3 = zero_like(m.eta), qf = zero_like(m.eta);
  if constexpr (tensor) {
    tt[0] = txx * txx + txy * txy + txz * txz;
    tt[1] = txx * txy + txy * tyy + txz * tyz;
    tt[2] = txx * txz + txy * tyz + txz * tzz;
    tt[3] = txy * txy + tyy * tyy + tyz * tyz;
    tt[4] = txy * txz + tyy * tyz + tyz * tzz;
    tt[5] = txz * txz + tyz * tyz + tzz * tzz;
    trT2 = tt[0] + tt[3] + tt[5];
    trT3 = tt[0] * txx + tt[3] * tyy + tt[5] * tzz + 2.0 * (tt[1] * txy + tt[2] * txz + tt[4] * tyz);
    tv[0] = txx * m.v1[0] + txy * m.v1[1] + txz * m.v1[2];
    tv[1] = txy * m.v1[0] + tyy * m.v1[1] + tyz * m.v1[2];
    tv[2] = txz * m.v1[0] + tyz * m.v1[1] + tzz * m.v1[2];
    qf = m.v1[0] * tv[0] + m.v1[1] * tv[1] + m.v1[2] * tv[2];
  }

  // Phi3 and its partials
  T p3, dp3_n2, dp3_v[3];
  const T n2 = m.n2;
  if constexpr (model == kRosenfeld) {
    p3 = INV_24PI * (n2 * n2 * n2 - 3.0 * n2 * dot11);
    dp3_n2 = INV_8PI * (n2 * n2 - dot11);
#pragma unroll
    for (int a = 0; a < 3; ++a) dp3_v[a] = -INV_4PI * n2 * m.v1[a];
  } else if constexpr (model == kRSLT) {
    if (val(n2) < 1e-30) {
      p3 = zero_like(n2);
      dp3_n2 = zero_like(n2);
  #pragma unroll
    for (int a = 0; a < 3; ++a) dp3_v[a] = zero_like(n2);
    } else {
      T xi = dot11 / (n2 * n2);
      if (val(xi) > 1.0) xi = cst<T>(1.0);  // std::min(xi, 1.0), models.hpp:210
      T q = 1.0 - xi;
      p3 = INV_36PI * n2 * n2 * n2 * q * q * q;
      dp3_n2 = INV_36PI * 3.0 * n2 * n2 * q * q * (1.0 + xi);
  #pragma unroll
    for (int a = 0; a < 3; ++a) dp3_v[a] = INV_36PI * (-6.0) * n2 * q * q * m.v1[a];
    }
  } else if constexpr (model == kWhiteBearI || model == kWhiteBearII) {
    p3 = INV_24PI * 3.0 * (n2 * trT2 - n2 * dot11 + qf - trT3);
    dp3_n2 = INV_24PI * 3.0 * (trT2 - dot11);
#pragma unroll
    for (int a = 0; a < 3; ++a) dp3_v[a] = INV_24PI * (-6.0 * n2 * m.v1[a] + 6.0 * tv[a]);
  } else {  // esFMT(A, B)
    T phi_a = n2 * n2 * n2 - 3.0 * n2 * dot11 + 3.0 * qf - trT3;
    T phi_b = n2 * n2 * n2 - 3.0 * n2 * trT2 + 2.0 * trT3;
    p3 = INV_24PI * (A * phi_a + B * phi_b);
    dp3_n2 = INV_24PI * (A * (3.0 * n2 * n2 - 3.0 * dot11) + B * (3.0 * n2 * n2 - 3.0 * trT2));
#pragma unroll
    for (int a = 0; a < 3; ++a) dp3_v[a] = INV_24PI * A * (-6.0 * n2 * m.v1[a] + 6.0 * tv[a]);
  }

  FVals<T> f = fmt_f<MODEL, T, FAST>(m.eta);
  if constexpr (ONE) {
    const T c2 = a1 * (n2 * n2 - dot11);
    const T n0 = a0 * n2;
    phi = -n0 * f.f1 + c2 * f.f2 + p3 * f.f3;
    dm.d_eta = -n0 * f.df1 + c2 * f.df2 + p3 * f.df3;
    dm.d_n0 = zero_like(m.eta);
    dm.d_n1 = zero_like(m.eta);
    dm.d_n2 = -a0 * f.f1 + (2.0 * a1) * n2 * f.f2 + dp3_n2 * f.f3;
    const T g = (-2.0 * a1) * f.f2;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dm.d_v0[a] = zero_like(m.eta);
      dm.d_v1[a] = g * m.v1[a] + dp3_v[a] * f.f3;
    }
  } else {
    T c2 = m.n1 * n2 - dot01;
    phi = -m.n0 * f.f1 + c2 * f.f2 + p3 * f.f3;
    dm.d_eta = -m.n0 * f.df1 + c2 * f.df2 + p3 * f.df3;
    dm.d_n0 = -f.f1;
    dm.d_n1 = n2 * f.f2;
    dm.d_n2 = m.n1 * f.f2 + dp3_n2 * f.f3;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dm.d_v0[a] = -m.v1[a] * f.f2;
      dm.d_v1[a] = -m.v0[a] * f.f2 + dp3_v[a] * f.f3;
    }
  }
  if constexpr (tensor) {
    // dPhi3/dT_ij (models.hpp:39-45, 348-357); T and TT symmetric
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (j < i) continue;
        const int c = tensor_index(i, j);
        T vv = m.v1[i] * m.v1[j];
        T d;
        if constexpr (model == kEsFMT) {
          d = INV_8PI * A * (vv - tt[c]) + INV_4PI * B * (-n2 * m.t[c] + tt[c]);
        } else {
          d = INV_8PI * (vv + 2.0 * n2 * m.t[c] - 3.0 * tt[c]);
        }
        dm.d_t[c] = d * f.f3;
      }
    }
  } else {
#pragma unroll
    for (int c = 0; c < 6; ++c) dm.d_t[c] = zero_like(m.eta);
  }
  return true;
}

}  // namespace cdft
