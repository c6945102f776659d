// staple.cuh -- the staple of a link, GaugeField.hpp:187-237 (3D :389-433,
// 2D :579-618) with the PTBC defect factors of PTBCGaugeField.hpp:232-277:
//   S = sum_{nu != mu} U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
//     + sum_{nu != mu} U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
// accumulated in the reference's order (all forward terms, then all backward).
#pragma once
#include "common.cuh"

namespace klft {

// DF = false compiles the defect handling out (lattices without a PTBC defect).
template <int NC, typename T, bool DF>
KLFT_D Mat<NC, T> load_link(const Links<NC, T> &U, const Geom &g, const Site &s, int mu, const Defect &df) {
  Mat<NC, T> m = U.load(site_lin(g, s), mu);
  if constexpr (DF) {
    if (df.active && in_defect(g, df, s, mu)) m = mscale(m, (T)defect_c(df));
  }
  return m;
}

// The nu loops stay rolled: the update kernels are instruction-fetch bound when
// the 4(Nd-1) products are all inlined next to the proposal code.
template <int NC, int ND, typename T, bool DF = false>
KLFT_D Mat<NC, T> staple(const Links<NC, T> &U, const Geom &g, const Site &x, int mu, const Defect &df) {
  Mat<NC, T> S = mzero<NC, T>();
  const Site xpmu = site_up(g, x, mu);
#pragma unroll 1
  for (int nu = 0; nu < ND; ++nu) {
    if (nu == mu) continue;
    const Site xpnu = site_up(g, x, nu);
    const Mat<NC, T> t = mul_nd(load_link<NC, T, DF>(U,g, xpmu, nu, df), load_link<NC, T, DF>(U,g, xpnu, mu, df));
    madd(S, mul_nd(t, load_link<NC, T, DF>(U,g, x, nu, df)));
  }
#pragma unroll 1
  for (int nu = 0; nu < ND; ++nu) {
    if (nu == mu) continue;
    const Site xpmu_mnu = site_dn(g, xpmu, nu);
    const Site xmnu = site_dn(g, x, nu);
    const Mat<NC, T> t = mul_dd(load_link<NC, T, DF>(U,g, xpmu_mnu, nu, df), load_link<NC, T, DF>(U,g, xmnu, mu, df));
    madd(S, mul(t, load_link<NC, T, DF>(U,g, xmnu, nu, df)));
  }
  return S;
}

// SU(3) with links stored as two FP32 rows (the mixed form, no defect): every
// staple term is a product of three SU(3) links and so itself in SU(3), which
// lets most of its third rows come from the first two (row 2 = conj(row 0 x
// row 1)) instead of from products:
//   forward  A B^+ C^+ = A (C B)^+,  backward  D^+ E^+ G = (E D)^+ G,
// with C B and E D formed on their first two rows (C and E need no third row),
// completed, and each term formed on its first two rows and completed.  Same
// terms in the same order as staple(); rounding differs at FP32 level.
template <typename T> KLFT_D void complete_row2(Mat<3, T> &m) {
  m.e[2][0] = conj(m.e[0][1] * m.e[1][2] - m.e[0][2] * m.e[1][1]);
  m.e[2][1] = conj(m.e[0][2] * m.e[1][0] - m.e[0][0] * m.e[1][2]);
  m.e[2][2] = conj(m.e[0][0] * m.e[1][1] - m.e[0][1] * m.e[1][0]);
}
// rows 0, 1 of a b (a's third row is not read)
template <typename T> KLFT_D void mul_rows01(const Mat<3, T> &a, const Mat<3, T> &b, Mat<3, T> &c) {
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) c.e[i][j] = a.e[i][0] * b.e[0][j] + a.e[i][1] * b.e[1][j] + a.e[i][2] * b.e[2][j];
}
// rows 0, 1 of a b^+
template <typename T> KLFT_D void mul_nd_rows01(const Mat<3, T> &a, const Mat<3, T> &b, Mat<3, T> &c) {
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      c.e[i][j] = a.e[i][0] * conj(b.e[j][0]) + a.e[i][1] * conj(b.e[j][1]) + a.e[i][2] * conj(b.e[j][2]);
}
// rows 0, 1 of a^+ b
template <typename T> KLFT_D void mul_dn_rows01(const Mat<3, T> &a, const Mat<3, T> &b, Mat<3, T> &c) {
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      c.e[i][j] = conj(a.e[0][i]) * b.e[0][j] + conj(a.e[1][i]) * b.e[1][j] + conj(a.e[2][i]) * b.e[2][j];
}

// The two-row staple with mu fixed at compile time and the nu loops unrolled:
// each link pass compiles its own site steps and can issue the loads of
// several terms ahead of their products.  1.62 -> 1.50 ms per SU(3) 32^4 sweep
// against a run-time mu (1.56 with the nu loops rolled).
template <int ND, int MU>
KLFT_D Mat<3, float> staple_su3_2row_ct(const Links<3, float> &U, const Geom &g, const Site &x) {
  Mat<3, float> S = mzero<3, float>();
  const Site xpmu = site_up(g, x, MU);
#pragma unroll
  for (int nu = 0; nu < ND; ++nu) {
    if (nu == MU) continue;
    const Site xpnu = site_up(g, x, nu);
    Mat<3, float> cb, f;
    mul_rows01(U.load_rows01(site_lin(g, x), nu), U.load(site_lin(g, xpnu), MU), cb);
    complete_row2(cb);
    mul_nd_rows01(U.load_rows01(site_lin(g, xpmu), nu), cb, f);
    complete_row2(f);
    madd(S, f);
  }
#pragma unroll
  for (int nu = 0; nu < ND; ++nu) {
    if (nu == MU) continue;
    const Site xpmu_mnu = site_dn(g, xpmu, nu);
    const Site xmnu = site_dn(g, x, nu);
    Mat<3, float> ed, f;
    mul_rows01(U.load_rows01(site_lin(g, xmnu), MU), U.load(site_lin(g, xpmu_mnu), nu), ed);
    complete_row2(ed);
    mul_dn_rows01(ed, U.load(site_lin(g, xmnu), nu), f);
    complete_row2(f);
    madd(S, f);
  }
  return S;
}

// The same staple with mu fixed at compile time and the nu loops unrolled: the
// same products in the same order, but every site step and index folds to a few
// integer operations.  For kernels without proposal code (the HMC force), where
// the unrolled products fit the instruction cache.
// DF: the PTBC defect factors as in staple() (only links of direction 0 can
// carry one, which the compiled direction makes visible to the compiler).
template <int NC, int ND, int MU, typename T, bool DF = false>
KLFT_D Mat<NC, T> staple_ct(const Links<NC, T> &U, const Geom &g, const Site &x, const Defect &df = Defect{}) {
  Mat<NC, T> S = mzero<NC, T>();
  const Site xpmu = site_up(g, x, MU);
#pragma unroll
  for (int nu = 0; nu < ND; ++nu) {
    if (nu == MU) continue;
    const Site xpnu = site_up(g, x, nu);
    const Mat<NC, T> t = mul_nd(load_link<NC, T, DF>(U, g, xpmu, nu, df), load_link<NC, T, DF>(U, g, xpnu, MU, df));
    madd(S, mul_nd(t, load_link<NC, T, DF>(U, g, x, nu, df)));
  }
#pragma unroll
  for (int nu = 0; nu < ND; ++nu) {
    if (nu == MU) continue;
    const Site xpmu_mnu = site_dn(g, xpmu, nu);
    const Site xmnu = site_dn(g, x, nu);
    const Mat<NC, T> t =
        mul_dd(load_link<NC, T, DF>(U, g, xpmu_mnu, nu, df), load_link<NC, T, DF>(U, g, xmnu, MU, df));
    madd(S, mul(t, load_link<NC, T, DF>(U, g, xmnu, nu, df)));
  }
  return S;
}

// staple_ct for a run-time mu (uniform across a warp in the callers)
template <int NC, int ND, typename T>
KLFT_D Mat<NC, T> staple_dispatch(const Links<NC, T> &U, const Geom &g, const Site &x, int mu) {
  if (mu == 0) return staple_ct<NC, ND, 0, T>(U, g, x);
  if (mu == 1) return staple_ct<NC, ND, 1, T>(U, g, x);
  if constexpr (ND > 2) {
    if (mu == 2) return staple_ct<NC, ND, 2, T>(U, g, x);
  }
  if constexpr (ND > 3) return staple_ct<NC, ND, 3, T>(U, g, x);
  return staple_ct<NC, ND, ND - 1, T>(U, g, x);
}

// Site of a class-blocked index lin = sub * Vh + hidx in 32-bit arithmetic
// (lattices with Vh < 2^31).
KLFT_D Site site_from_lin32(const Geom &g, unsigned lin) {
  Site s;
  const unsigned vh = (unsigned)g.Vh;
  const unsigned sub = lin / vh;
  unsigned hidx = lin - sub * vh;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const unsigned hd = (unsigned)g.H[d];
    const unsigned q = hidx / hd;
    s.set_b(d, (int)((sub >> d) & 1u));
    s.set_h(d, (int)(hidx - q * hd));
    hidx = q;
  }
  return s;
}

}  // namespace klft
