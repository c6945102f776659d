// group.cuh -- group-specific device math: Metropolis proposals, Haar-random
// links, and the Lie-algebra maps used by HMC (the SU(3) exponential is in
// expprop.cuh).
#pragma once
#include "common.cuh"
#include "expprop.cuh"

namespace klft {

constexpr double KPI = 3.141592653589793;
constexpr double K2PI = 6.283185307179586;

enum Proposal : int { PROPOSAL_REFERENCE = 0, PROPOSAL_EXP = 1 };

// ------------------------------------------------------------------ proposals
// U(1): exp(i phi), phi uniform in [-delta*pi, delta*pi]   (SUN.hpp:163-171)
template <typename T> KLFT_D Mat<1, T> propose(Stream &g, const Mat<1, T> *, double delta, int, double) {
  const double phi = g.drand(-delta * KPI, delta * KPI);
  Mat<1, T> r;
  r.e[0][0] = mk<T>((T)cos(phi), (T)sin(phi));
  return r;
}
// SU(2): cos(a) + i sin(a) n.sigma  (SUN.hpp:174-189)
template <typename T> KLFT_D Mat<2, T> propose(Stream &g, const Mat<2, T> *, double delta, int, double) {
  const T alpha = (T)g.drand(0.0, delta * 2 * KPI);
  const T u = (T)g.drand(-1.0, 1.0);
  const T theta = (T)g.drand(0.0, 2.0 * KPI);
  const T salpha = sin(alpha);
  const T su = sqrt(T(1) - u * u);
  const T n1 = su * sin(theta);
  const T n2 = su * cos(theta);
  Mat<2, T> r;
  r.e[0][0] = mk<T>(cos(alpha), u * salpha);
  r.e[0][1] = mk<T>(n1 * salpha, n2 * salpha);
  r.e[1][0] = mk<T>(-r.e[0][1].re, r.e[0][1].im);
  r.e[1][1] = mk<T>(r.e[0][0].re, -r.e[0][0].im);
  return r;
}
// SU(3): reference Gram-Schmidt proposal (SUN.hpp:192-251); the exp(i eps H)
// proposal has its own fixed-position stream (expprop.cuh).
template <typename T> KLFT_D Mat<3, T> propose(Stream &g, const Mat<3, T> *, double delta, int, double) {
  Mat<3, T> r;
  T r1[6], r2[6], norm, fact;
  cx<T> z1[3], z2[3], z3[3], z;
  // The rejection loops of the reference end once a draw has nonzero norm; they
  // are bounded here (the host rejects delta <= 0, for which they never end).
  for (int tries = 0; tries < 64; ++tries) {
#pragma unroll
    for (int i = 0; i < 6; ++i) r1[i] = (T)g.drand(0.0, delta);
    norm = sqrt(r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2] + r1[3] * r1[3] + r1[4] * r1[4] + r1[5] * r1[5]);
    if (T(1) != (T(1) + norm)) break;
  }
  fact = T(1) / norm;
  z1[0] = fact * mk<T>(r1[0], r1[1]);
  z1[1] = fact * mk<T>(r1[2], r1[3]);
  z1[2] = fact * mk<T>(r1[4], r1[5]);
  for (int outer = 0; outer < 64; ++outer) {
    for (int tries = 0; tries < 64; ++tries) {
#pragma unroll
      for (int i = 0; i < 6; ++i) r2[i] = (T)g.drand(0.0, delta);
      norm = sqrt(r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2] + r2[3] * r2[3] + r2[4] * r2[4] + r2[5] * r2[5]);
      if (T(1) != (T(1) + norm)) break;
    }
    fact = T(1) / norm;
    z2[0] = fact * mk<T>(r2[0], r2[1]);
    z2[1] = fact * mk<T>(r2[2], r2[3]);
    z2[2] = fact * mk<T>(r2[4], r2[5]);
    z = conj(z1[0]) * z2[0] + conj(z1[1]) * z2[1] + conj(z1[2]) * z2[2];
    z2[0] -= z * z1[0];
    z2[1] -= z * z1[1];
    z2[2] -= z * z1[2];
    norm = sqrt(z2[0].re * z2[0].re + z2[0].im * z2[0].im + z2[1].re * z2[1].re + z2[1].im * z2[1].im +
                z2[2].re * z2[2].re + z2[2].im * z2[2].im);
    if (T(1) != (T(1) + norm)) break;
  }
  fact = T(1) / norm;
  z2[0] = z2[0] * fact;
  z2[1] = z2[1] * fact;
  z2[2] = z2[2] * fact;
  z3[0] = conj((z1[1] * z2[2]) - (z1[2] * z2[1]));
  z3[1] = conj((z1[2] * z2[0]) - (z1[0] * z2[2]));
  z3[2] = conj((z1[0] * z2[1]) - (z1[1] * z2[0]));
#pragma unroll
  for (int j = 0; j < 3; ++j) { r.e[0][j] = z1[j]; r.e[1][j] = z2[j]; r.e[2][j] = z3[j]; }
  return r;
}

// ------------------------------------------------------------------ hot start
template <typename T> KLFT_D Mat<1, T> haar(Stream &g, const Mat<1, T> *) {
  const double phi = g.drand(-KPI, KPI);
  Mat<1, T> m;
  m.e[0][0] = mk<T>((T)cos(phi), (T)sin(phi));
  return m;
}
template <typename T> KLFT_D Mat<2, T> haar(Stream &g, const Mat<2, T> *) {
  double q[4];
  g.gauss2(q[0], q[1]);
  g.gauss2(q[2], q[3]);
  const double n = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
#pragma unroll
  for (int k = 0; k < 4; ++k) q[k] /= n;
  Mat<2, T> m;
  m.e[0][0] = mk<T>((T)q[0], (T)q[3]);
  m.e[0][1] = mk<T>((T)q[2], (T)q[1]);
  m.e[1][0] = mk<T>((T)-q[2], (T)q[1]);
  m.e[1][1] = mk<T>((T)q[0], (T)-q[3]);
  return m;
}
template <typename T> KLFT_D Mat<3, T> haar(Stream &g, const Mat<3, T> *) {
  cx<double> r0[3], r1[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) { double a, b; g.gauss2(a, b); r0[j] = mk(a, b); }
#pragma unroll
  for (int j = 0; j < 3; ++j) { double a, b; g.gauss2(a, b); r1[j] = mk(a, b); }
  const double n0 = sqrt(r0[0].re * r0[0].re + r0[0].im * r0[0].im + r0[1].re * r0[1].re + r0[1].im * r0[1].im +
                         r0[2].re * r0[2].re + r0[2].im * r0[2].im);
#pragma unroll
  for (int j = 0; j < 3; ++j) r0[j] = cdiv(r0[j], n0);
  const cx<double> z = conj(r0[0]) * r1[0] + conj(r0[1]) * r1[1] + conj(r0[2]) * r1[2];
#pragma unroll
  for (int j = 0; j < 3; ++j) r1[j] -= z * r0[j];
  const double n1 = sqrt(r1[0].re * r1[0].re + r1[0].im * r1[0].im + r1[1].re * r1[1].re + r1[1].im * r1[1].im +
                         r1[2].re * r1[2].re + r1[2].im * r1[2].im);
#pragma unroll
  for (int j = 0; j < 3; ++j) r1[j] = cdiv(r1[j], n1);
  cx<double> r2[3];
  r2[0] = conj(r0[1] * r1[2] - r0[2] * r1[1]);
  r2[1] = conj(r0[2] * r1[0] - r0[0] * r1[2]);
  r2[2] = conj(r0[0] * r1[1] - r0[1] * r1[0]);
  Mat<3, T> m;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    m.e[0][j] = mk<T>((T)r0[j].re, (T)r0[j].im);
    m.e[1][j] = mk<T>((T)r1[j].re, (T)r1[j].im);
    m.e[2][j] = mk<T>((T)r2[j].re, (T)r2[j].im);
  }
  return m;
}

// ------------------------------------------------------------------ Lie algebra (HMC)
template <int N> struct Alg { static constexpr int n = N == 1 ? 1 : (N == 2 ? 3 : 8); };

// Adj(M): U(1) Im M (AdjointGroup.hpp:114-117); SU(2) (2 Im M01, 2 Re M01, 2 Im M00)
// (AdjointGroup.hpp:13-19); SU(3) Im Tr(lambda_a M), the same projection with the
// Gell-Mann generators.
template <typename T> KLFT_D void adjoint(const Mat<1, T> &M, T *v) { v[0] = M.e[0][0].im; }
template <typename T> KLFT_D void adjoint(const Mat<2, T> &M, T *v) {
  v[0] = T(2) * M.e[0][1].im;
  v[1] = T(2) * M.e[0][1].re;
  v[2] = T(2) * M.e[0][0].im;
}
template <typename T> KLFT_D void adjoint(const Mat<3, T> &M, T *v) {
  const T r3 = T(1) / sqrt(T(3));
  v[0] = M.e[1][0].im + M.e[0][1].im;            // lambda_1
  v[1] = -M.e[1][0].re + M.e[0][1].re;           // lambda_2
  v[2] = M.e[0][0].im - M.e[1][1].im;            // lambda_3
  v[3] = M.e[2][0].im + M.e[0][2].im;            // lambda_4
  v[4] = -M.e[2][0].re + M.e[0][2].re;           // lambda_5
  v[5] = M.e[2][1].im + M.e[1][2].im;            // lambda_6
  v[6] = -M.e[2][1].re + M.e[1][2].re;           // lambda_7
  v[7] = (M.e[0][0].im + M.e[1][1].im - T(2) * M.e[2][2].im) * r3;  // lambda_8
}

// exp map U <- exp(t P) U: U(1) e^{i t p} (AdjointGroup.hpp:170-173); SU(2)
// cos|a| + i sin|a| n.sigma, a = t p (AdjointGroup.hpp:98-105, with exp(0) = 1);
// SU(3) exp(i t sum_a p_a lambda_a).
template <typename T> KLFT_D Mat<1, T> expmap(const T *p, T t, const Mat<1, T> *) {
  Mat<1, T> m;
  m.e[0][0] = mk<T>(cos(t * p[0]), sin(t * p[0]));
  return m;
}
template <typename T> KLFT_D Mat<2, T> expmap(const T *p, T t, const Mat<2, T> *) {
  const T a0 = t * p[0], a1 = t * p[1], a2 = t * p[2];
  const T alpha = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
  if (alpha == T(0)) return mident<2, T>();
  const T n0 = a0 / alpha, n1 = a1 / alpha, n2 = a2 / alpha;
  const T sa = sin(alpha), ca = cos(alpha);
  Mat<2, T> m;
  m.e[0][0] = mk<T>(ca, n2 * sa);
  m.e[0][1] = mk<T>(n1 * sa, n0 * sa);
  m.e[1][0] = mk<T>(-n1 * sa, n0 * sa);
  m.e[1][1] = mk<T>(ca, -n2 * sa);
  return m;
}
template <typename T> KLFT_D Mat<3, T> expmap(const T *p, T t, const Mat<3, T> *) {
  const XMat<T> x = expi_gellmann<T>(p, t);
  Mat<3, T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.e[i][j] = mk<T>(x.re[i][j], x.im[i][j]);
  return m;
}

}  // namespace klft
