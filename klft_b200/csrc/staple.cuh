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

}  // namespace klft
