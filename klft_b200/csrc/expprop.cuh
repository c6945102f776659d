// expprop.cuh -- the SU(3) proposal X = exp(i eps H) of the Metropolis sweep,
// H = sum_a h_a lambda_a / 2 with h_a Gaussian (no counterpart in the
// reference, whose SU(3) proposal is the Gram-Schmidt generator of
// SUN.hpp:192-251).
//
// Random numbers: hit h of a site (h = mu*nHits + hit) reads Philox block h of
// sub-stream 0 of the (sweep, site) stream; each 32-bit word gives two 16-bit
// uniforms u = (k + 1/2) 2^-16 (low half, then high half), one Box-Muller pair,
// so one block gives the eight Gaussians of a proposal.  Its accept uniform is
// word h mod 4 of block h / 4 of sub-stream 1, (w + 1/2) 2^-32.  A proposal
// never depends on earlier accept decisions.  The 16-bit grid is symmetric
// under u -> u + 1/2, so every h_a is symmetric and X and X^-1 are proposed
// with equal probability (detailed balance of the proposal).
//
// The exponential is evaluated in the Cayley-Hamilton basis (1, Q, Q^2),
// Q = (eps/2) sum_a h_a lambda_a, with the Gell-Mann structure written out:
// Q^2, Tr Q^2 / 2 and det Q come straight from the eight coefficients.  The
// arithmetic is written once for the value type V (double: FP64 form, float:
// mixed form) through the small v* helpers.
#pragma once
#include "common.cuh"

namespace klft {

// ------------------------------------------------------------------ arithmetic helpers
KLFT_D double vfma(double a, double b, double c) { return fma(a, b, c); }
KLFT_D double vmul(double a, double b) { return a * b; }
KLFT_D double vadd(double a, double b) { return a + b; }
KLFT_D double vsub(double a, double b) { return a - b; }
KLFT_D float vfma(float a, float b, float c) { return fmaf(a, b, c); }
KLFT_D float vmul(float a, float b) { return a * b; }
KLFT_D float vadd(float a, float b) { return a + b; }
KLFT_D float vsub(float a, float b) { return a - b; }
template <typename V> KLFT_D V splat(double c);
template <> KLFT_D double splat<double>(double c) { return c; }
template <> KLFT_D float splat<float>(double c) { return (float)c; }
KLFT_D double vmax(double a) { return a; }
KLFT_D float vmax(float a) { return a; }

// Terms of the coefficient series: |lambda| <= 1 after scaling, so 1/12! < 3e-9
// in FP32 and 1/19! < 1e-17 in FP64.
template <typename V> struct SeriesTerms { static constexpr int n = 12; };
template <> struct SeriesTerms<double> { static constexpr int n = 19; };

template <typename V> struct XMat { V re[3][3], im[3][3]; };

// exp(i Q), Q = s sum_a h_a lambda_a (Gell-Mann, a = 1..8; h[a-1] holds h_a).
// Cayley-Hamilton: Q^3 = c1 Q + c0 with c1 = Tr Q^2 / 2 = sum_a (s h_a)^2 and
// c0 = det Q, so Q^n = a_n + b_n Q + d_n Q^2 with (a, b, d)_{n+1} =
// (d c0, a + d c1, b), and exp(iQ) = f0 + f1 Q + f2 Q^2 with
// f = sum_n i^n / n! (a_n, b_n, d_n).  Arguments with c1 > 3/4 (an eigenvalue
// possibly above 1: |lambda|^2 <= 4 c1 / 3) are scaled by 2^-k and the result
// squared k times in coefficient space:
//   (f0 + f1 Q + f2 Q^2)^2 = (f0^2 + 2 f1 f2 c0) + (2 f0 f1 + 2 f1 f2 c1 + f2^2 c0) Q
//                          + (f1^2 + 2 f0 f2 + f2^2 c1) Q^2.
template <typename V> KLFT_D XMat<V> expi_gellmann(const V h[8], V s) {
  V a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = vmul(s, h[k]);
  // Q: diagonal (d0, d1, d2) real; Q01 = a1 - i a2, Q02 = a4 - i a5, Q12 = a6 - i a7
  const V e8 = vmul(splat<V>(0.57735026918962576451), a[7]);
  const V d0 = vadd(e8, a[2]), d1 = vsub(e8, a[2]), d2 = vmul(splat<V>(-2.0), e8);
  const V n01 = vfma(a[0], a[0], vmul(a[1], a[1]));
  const V n02 = vfma(a[3], a[3], vmul(a[4], a[4]));
  const V n12 = vfma(a[5], a[5], vmul(a[6], a[6]));
  // c1 = Tr Q^2 / 2 = sum a_k^2, c0 = det Q = d0 d1 d2 + 2 Re(Q01 Q12 conj(Q02))
  // - d0 n12 - d1 n02 - d2 n01 (Q^2 itself is formed after the series, so that
  // its entries are not live while the series runs)
  const V u = vsub(vmul(a[0], a[5]), vmul(a[1], a[6]));   // Re Q01 Q12
  const V v = vfma(a[0], a[6], vmul(a[1], a[5]));          // -Im Q01 Q12
  V c1 = vmul(a[0], a[0]);
#pragma unroll
  for (int k = 1; k < 8; ++k) c1 = vfma(a[k], a[k], c1);
  const V re3 = vfma(u, a[3], vmul(v, a[4]));
  V c0 = vmul(vmul(d0, d1), d2);
  c0 = vfma(splat<V>(2.0), re3, c0);
  c0 = vsub(c0, vfma(d0, n12, vfma(d1, n02, vmul(d2, n01))));
  int sq = 0;
  V cs1 = c1, cs0 = c0, scale = splat<V>(1.0);
  float big = (float)vmax(c1);
  while (big > 0.75f && sq < 64) {  // halve Q: c1 / 4, c0 / 8
    cs1 = vmul(cs1, splat<V>(0.25));
    cs0 = vmul(cs0, splat<V>(0.125));
    scale = vmul(scale, splat<V>(0.5));
    big *= 0.25f;
    ++sq;
  }
  // Taylor sum of exp(i Q'), Q' = scale Q, in the basis (1, Q', Q'^2)
  V ta = splat<V>(1.0), tb = splat<V>(0.0), td = splat<V>(0.0);
  V f0r = splat<V>(1.0), f0i = splat<V>(0.0), f1r = splat<V>(0.0), f1i = splat<V>(0.0), f2r = splat<V>(0.0),
    f2i = splat<V>(0.0);
  double fact = 1.0;
#pragma unroll
  for (int n = 1; n < SeriesTerms<V>::n; ++n) {
    const V an = vmul(td, cs0), bn = vfma(td, cs1, ta), dn = tb;
    ta = an;
    tb = bn;
    td = dn;
    fact /= (double)n;
    const V cf = splat<V>(((n >> 1) & 1) ? -fact : fact);  // i^n: 1, i, -1, -i
    if (n & 1) {
      f0i = vfma(cf, ta, f0i);
      f1i = vfma(cf, tb, f1i);
      f2i = vfma(cf, td, f2i);
    } else {
      f0r = vfma(cf, ta, f0r);
      f1r = vfma(cf, tb, f1r);
      f2r = vfma(cf, td, f2r);
    }
  }
  for (int k = 0; k < sq; ++k) {
    // complex f12 = f1 f2, f22 = f2^2
    const V f12r = vsub(vmul(f1r, f2r), vmul(f1i, f2i)), f12i = vfma(f1r, f2i, vmul(f1i, f2r));
    const V f22r = vsub(vmul(f2r, f2r), vmul(f2i, f2i)), f22i = vmul(splat<V>(2.0), vmul(f2r, f2i));
    const V tc0 = vmul(splat<V>(2.0), cs0), tc1 = vmul(splat<V>(2.0), cs1);
    const V g0r = vfma(f12r, tc0, vsub(vmul(f0r, f0r), vmul(f0i, f0i)));
    const V g0i = vfma(f12i, tc0, vmul(splat<V>(2.0), vmul(f0r, f0i)));
    const V g1r = vfma(f22r, cs0, vfma(f12r, tc1, vmul(splat<V>(2.0), vsub(vmul(f0r, f1r), vmul(f0i, f1i)))));
    const V g1i = vfma(f22i, cs0, vfma(f12i, tc1, vmul(splat<V>(2.0), vfma(f0r, f1i, vmul(f0i, f1r)))));
    const V g2r = vfma(f22r, cs1, vfma(splat<V>(2.0), vsub(vmul(f0r, f2r), vmul(f0i, f2i)),
                                       vsub(vmul(f1r, f1r), vmul(f1i, f1i))));
    const V g2i = vfma(f22i, cs1, vfma(splat<V>(2.0), vfma(f0r, f2i, vmul(f0i, f2r)),
                                       vmul(splat<V>(2.0), vmul(f1r, f1i))));
    f0r = g0r; f0i = g0i; f1r = g1r; f1i = g1i; f2r = g2r; f2i = g2i;
    cs1 = vmul(cs1, splat<V>(4.0));
    cs0 = vmul(cs0, splat<V>(8.0));
  }
  // back to the basis (1, Q, Q^2): Q' = scale Q
  if (sq) {
    const V sc2 = vmul(scale, scale);
    f1r = vmul(f1r, scale);
    f1i = vmul(f1i, scale);
    f2r = vmul(f2r, sc2);
    f2i = vmul(f2i, sc2);
  }
  // Q^2 (hermitian): diagonal and upper triangle
  const V s00 = vfma(d0, d0, vadd(n01, n02));
  const V s11 = vfma(d1, d1, vadd(n01, n12));
  const V s22 = vfma(d2, d2, vadd(n02, n12));
  const V te8 = vadd(e8, e8), am = vsub(a[2], e8), ap = vadd(e8, a[2]);
  // (Q^2)_01 = -d2 Q01 + Q02 conj(Q12)
  const V s01r = vfma(te8, a[0], vfma(a[3], a[5], vmul(a[4], a[6])));
  const V s01i = vsub(vsub(vmul(a[3], a[6]), vmul(a[4], a[5])), vmul(te8, a[1]));
  // (Q^2)_02 = -d1 Q02 + Q01 Q12
  const V s02r = vfma(am, a[3], u);
  const V s02i = vsub(splat<V>(0.0), vfma(am, a[4], v));
  // (Q^2)_12 = conj(Q01) Q02 - d0 Q12
  const V s12r = vsub(vfma(a[0], a[3], vmul(a[1], a[4])), vmul(ap, a[5]));
  const V s12i = vfma(ap, a[6], vsub(vmul(a[1], a[3]), vmul(a[0], a[4])));
  XMat<V> X;
  // diagonal: f0 + f1 d_i + f2 (Q^2)_ii
  const V dd[3] = {d0, d1, d2}, ss[3] = {s00, s11, s22};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    X.re[i][i] = vfma(f2r, ss[i], vfma(f1r, dd[i], f0r));
    X.im[i][i] = vfma(f2i, ss[i], vfma(f1i, dd[i], f0i));
  }
  // off-diagonal pairs: with P = Re(f1) Q_ij + Re(f2) Q2_ij and N = Im(f1) Q_ij + Im(f2) Q2_ij,
  // X_ij = P + i N and X_ji = conj(P) + i conj(N)
  const V qr[3] = {a[0], a[3], a[5]};
  const V qi[3] = {vmul(splat<V>(-1.0), a[1]), vmul(splat<V>(-1.0), a[4]), vmul(splat<V>(-1.0), a[6])};
  const V sr[3] = {s01r, s02r, s12r}, si[3] = {s01i, s02i, s12i};
  const int I[3] = {0, 0, 1}, J[3] = {1, 2, 2};
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const V Pr = vfma(f2r, sr[p], vmul(f1r, qr[p])), Pi = vfma(f2r, si[p], vmul(f1r, qi[p]));
    const V Nr = vfma(f2i, sr[p], vmul(f1i, qr[p])), Ni = vfma(f2i, si[p], vmul(f1i, qi[p]));
    X.re[I[p]][J[p]] = vsub(Pr, Ni);
    X.im[I[p]][J[p]] = vadd(Pi, Nr);
    X.re[J[p]][I[p]] = vadd(Pr, Ni);
    X.im[J[p]][I[p]] = vsub(Nr, Pi);
  }
  return X;
}

// Box-Muller pair from the two 16-bit halves of one stream word,
// u = (k + 1/2) 2^-16; (r cos 2 pi u_b, r sin 2 pi u_b), r = sqrt(-2 ln u_a).
// FP64: each half takes one of 2^16 values, so r, cos and sin are read from a
// table built on the host (bm_table(): r at [k], (cos, sin) at 2^16 + 2 k), the
// same expressions the oracle evaluates, instead of FP64 log / sqrt / sincos on
// the device (those cost about 30 % of an FP64 sweep).
constexpr int BM_TAB = 1 << 16;
KLFT_D void box_muller16(uint32_t w, double &g0, double &g1, const double *bm) {
  const double r = __ldg(bm + (w & 0xFFFFu));
  const double2 cs = __ldg((const double2 *)(bm + BM_TAB) + (w >> 16));
  g0 = r * cs.x;
  g1 = r * cs.y;
}
// FP32: the halves become floats in [1, 2) through their bit patterns (exact),
// SFU log, rsqrt and sincos; cos/sin(2 pi u) = -cos/sin(2 pi (u - 1/2)) keeps
// the SFU argument in [-pi, pi].
KLFT_D void box_muller16(uint32_t w, float &g0, float &g1) {
  const float ua = __int_as_float(0x3F800000u | ((w << 7) & 0x007FFF80u)) - (1.0f - 0x1.0p-17f);
  const float ub = __int_as_float(0x3F800000u | ((w >> 9) & 0x007FFF80u)) - (1.0f - 0x1.0p-17f);
  const float q = -2.0f * __logf(ua);
  const float r = q > 0.0f ? q * rsqrtf(q) : 0.0f;
  float sn, cs;
  __sincosf(6.28318530717958648f * (ub - 0.5f), &sn, &cs);
  g0 = -r * cs;
  g1 = -r * sn;
}

// Stream positions of the exp(i eps H) proposal of one site and sweep.
struct ExpHitStream {
  uint32_t k0, k1, site, step;
  const double *bm;  // Box-Muller table of the FP64 form (bm_table()); unused in FP32
  KLFT_D void block(uint32_t b, uint32_t w[4], uint32_t sub = 0) const {
    w[0] = b; w[1] = site; w[2] = step; w[3] = (KIND_METROPOLIS << 24) | sub;
    philox4x32_10(w, k0, k1);
  }
  // the eight Gaussians of hit h
  template <typename T> KLFT_D void gauss8(uint32_t h, T g[8]) const {
    uint32_t w[4];
    block(h, w);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if constexpr (sizeof(T) == 8) box_muller16(w[k], g[2 * k], g[2 * k + 1], bm);
      else box_muller16(w[k], g[2 * k], g[2 * k + 1]);
    }
  }
  KLFT_D void accept_block(uint32_t h, uint32_t w[4]) const { block(h >> 2, w, 1); }
};

KLFT_D double accept_word(const uint32_t w[4], uint32_t h) {
  const uint32_t j = h & 3;
  const uint32_t x = j == 0 ? w[0] : (j == 1 ? w[1] : (j == 2 ? w[2] : w[3]));
  return ((double)x + 0.5) * 0x1.0p-32;
}

// X of one hit as a matrix of T (T = double or float)
template <typename T> KLFT_D Mat<3, T> exp_proposal(const ExpHitStream &hs, uint32_t h, T half_eps) {
  T g[8];
  hs.gauss8<T>(h, g);
  const XMat<T> x = expi_gellmann<T>(g, half_eps);
  Mat<3, T> X;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) X.e[i][j] = mk<T>(x.re[i][j], x.im[i][j]);
  return X;
}

}  // namespace klft
