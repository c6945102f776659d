// metropolis_site.cuh -- the per-site Metropolis update shared by the
// single-lattice pass kernels (metropolis.cu) and the multi-chain batch kernels
// (batch.cu).
//
// Semantics follow MetropolisGaugeField::operator() (Metropolis.hpp:73-113): a
// thread owns one site of a parity class and updates its Nd links in order
// mu = 0..Nd-1; per link the staple is formed once, then nHits proposals
// U' = U r are accepted with probability min(1, exp(-dS)),
// dS = -(beta/Nc) Re Tr[(U' - U) S], and an accepted link is stored
// reunitarised (restoreSUN).
//
// Per-hit cost: with M = S U, Re Tr(U r S) = Re Tr(r M) needs only the diagonal
// of r M.  SU(3) reference proposals (a few per cent accepted) rebuild U r and M
// on acceptance; U(1)/SU(2) and the exp(i eps H) proposals, accepted on
// ~30-70 % of hits (so every warp runs the accept branch on nearly every hit),
// accumulate the accepted proposals into one matrix A instead and need one
// product per hit (see site_update_ref and site_update_exp).
//
// Random numbers: the reference proposals (U(1), SU(2), the SU(3)
// Gram-Schmidt generator) consume the site's sequential Philox stream in the
// order the reference functor consumes its generator.  The exp(i eps H)
// proposal (no reference counterpart) reads fixed stream positions per hit (see
// ExpHitStream), so a proposal does not depend on earlier accept decisions.
// Neither depends on the launch shape.
#pragma once
#include "group.cuh"
#include "kernels.cuh"
#include "staple.cuh"

namespace klft {

// Fixed-position stream of the exp(i eps H) proposal: hit h of a site
// (h = mu*nHits + hit) uses Philox blocks 2h, 2h+1 of sub-stream 0 (eight
// 32-bit uniforms u = (w + 1/2) 2^-32 for four Box-Muller pairs) and word h mod 4
// of block h / 4 of sub-stream 1 for its accept uniform (w + 1/2) 2^-32, so one
// block serves the accept decisions of four hits.
struct ExpHitStream {
  uint32_t k0, k1, site, step;
  KLFT_D void block(uint32_t b, uint32_t w[4], uint32_t sub = 0) const {
    w[0] = b; w[1] = site; w[2] = step; w[3] = (KIND_METROPOLIS << 24) | sub;
    philox4x32_10(w, k0, k1);
  }
  KLFT_D void accept_block(uint32_t h, uint32_t w[4]) const { block(h >> 2, w, 1); }
};

KLFT_D double accept_word(const uint32_t w[4], uint32_t h) {
  const uint32_t j = h & 3;
  const uint32_t x = j == 0 ? w[0] : (j == 1 ? w[1] : (j == 2 ? w[2] : w[3]));
  return ((double)x + 0.5) * 0x1.0p-32;
}

KLFT_D void box_muller(uint32_t wa, uint32_t wb, double &g0, double &g1) {
  const double ua = ((double)wa + 0.5) * 0x1.0p-32, ub = ((double)wb + 0.5) * 0x1.0p-32;
  const double r = sqrt(-2.0 * log(ua));
  double s, c;
  sincospi(2.0 * ub, &s, &c);
  g0 = r * c;
  g1 = r * s;
}
// Mixed form: SFU log, rsqrt and sincos.  cos/sin(2 pi u) = -cos/sin(2 pi (u - 1/2))
// keeps the SFU argument in [-pi, pi]; ua rounds to 1 for the largest words,
// where the radius is 0.
KLFT_D void box_muller(uint32_t wa, uint32_t wb, float &g0, float &g1) {
  const float ua = fmaf((float)wa, 0x1.0p-32f, 0x1.0p-33f), ub = fmaf((float)wb, 0x1.0p-32f, 0x1.0p-33f);
  const float q = -2.0f * __logf(ua);
  const float r = q > 0.0f ? q * rsqrtf(q) : 0.0f;
  float s, c;
  __sincosf(6.28318530717958648f * (ub - 0.5f), &s, &c);
  g0 = -r * c;
  g1 = -r * s;
}

// X = exp(i eps H) of one hit from its eight stream words (blocks 2h, 2h+1)
template <typename T>
KLFT_D Mat<3, T> exp_proposal_w(const uint32_t (&w)[8], T half_eps) {
  T g[8];
#pragma unroll
  for (int k = 0; k < 4; ++k) box_muller(w[2 * k], w[2 * k + 1], g[2 * k], g[2 * k + 1]);
  return expi_su3(gellmann_combo(g, half_eps));
}

template <int NC, typename T>
KLFT_D T retr_diag(const Mat<NC, T> &M) {
  T t = T(0);
#pragma unroll
  for (int i = 0; i < NC; ++i) t += M.e[i][i].re;
  return t;
}

// Block total of accepted hits -> one atomic per block.
KLFT_D void add_accepts(int nacc, unsigned long long *d_nacc) {
  __shared__ int red[32];
  const int v = warp_sum(nacc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    if (s) atomicAdd(d_nacc, (unsigned long long)s);
  }
}

// site t of parity class val: x_d = 2 h_d + bit_d, bit_d = (val >> (Nd-1-d)) & 1
KLFT_D Site pass_site(const Geom &g, long long t, int val, int nd) {
  Site x;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    x.set_h(d, (int)(t % g.H[d]));
    t /= g.H[d];
    x.set_b(d, d < nd ? (val >> (nd - 1 - d)) & 1 : 0);
  }
  return x;
}

template <typename T> struct MinBlocks { static constexpr int v = 4; };
template <> struct MinBlocks<double> { static constexpr int v = 2; };

// Reference proposals: sequential per-site stream, exactly as the reference consumes it.
template <int NC, int ND, typename T, bool DF>
KLFT_D int site_update_ref(const Links<NC, T> &U, const Geom &g, const Site &x, const MetroArgs &a, uint32_t sweep,
                           const Defect &df) {
  int nacc = 0;
  Stream rng(a.seed, a.chain, site_lex(g, x), sweep, KIND_METROPOLIS, 0);
  const long long lx = site_lin(g, x);
  const T bnc = (T)a.beta / (T)NC;
#pragma unroll 1
  for (int mu = 0; mu < ND; ++mu) {
    if (open_link(g, x, mu)) continue;
    const Mat<NC, T> S = staple<NC, ND, T, DF>(U, g, x, mu, df);
    const bool dlink = DF && df.active && in_defect(g, df, x, mu);
    if constexpr (NC <= 2) {
      // U(1), SU(2): accepted proposals accumulate into A = r_1 ... r_k, so the
      // current link is U0 A and Re Tr(U0 A r S) = Re Tr((A r) M0), M0 = S U0: one
      // product A r per hit, which is also the new A on acceptance (warps take the
      // accept branch on almost every hit).  The link is rebuilt as U0 A and
      // reunitarised once; the chain is the one of U <- restore(U r) per accepted
      // hit, with rounding-level differences.
      const Mat<NC, T> U0 = U.load(lx, mu);
      const Mat<NC, T> M0 = mul(S, U0);
      Mat<NC, T> A = mident<NC, T>();
      T trO = retr_diag(M0);
      bool changed = false;
#pragma unroll 1
      for (int hit = 0; hit < a.nhits; ++hit) {
        const Mat<NC, T> rr = propose<T>(rng, (const Mat<NC, T> *)nullptr, a.delta, PROPOSAL_REFERENCE, 0.0);
        const Mat<NC, T> Y = hit == 0 ? rr : mul(A, rr);
        const T tY = retr_mul(Y, M0);
        T dS = -bnc * (tY - trO);
        if (dlink) dS *= (T)defect_c(df);
        bool accept = dS < T(0);
        if (!accept) accept = rng.next() < (double)exp(-dS);
        if (accept) {
          A = Y;
          trO = tY;
          ++nacc;
          changed = true;
        }
      }
      if (changed) U.store(lx, mu, restore(mul(U0, A)));
      continue;
    }
    Mat<NC, T> Uo = U.load(lx, mu);
    Mat<NC, T> M = mul(S, Uo);
    T trO = retr_diag(M);
    bool changed = false;
#pragma unroll 1
    for (int hit = 0; hit < a.nhits; ++hit) {
      const Mat<NC, T> rr = propose<T>(rng, (const Mat<NC, T> *)nullptr, a.delta, PROPOSAL_REFERENCE, 0.0);
      T dS = -bnc * (retr_mul(rr, M) - trO);
      if (dlink) dS *= (T)defect_c(df);
      bool accept = dS < T(0);
      if (!accept) accept = rng.next() < (double)exp(-dS);
      if (accept) {
        Uo = restore(mul(Uo, rr));
        M = mul(S, Uo);
        trO = retr_diag(M);
        ++nacc;
        changed = true;
      }
    }
    if (changed) U.store(lx, mu, Uo);
  }
  return nacc;
}

// SU(3) exp(i eps H) proposals U' = X U at fixed stream positions.  The
// accepted proposals of a link accumulate into A = X_k ... X_1, so the current
// link is A U0 and, with M0 = U0 S formed once, a hit's action change needs
// Re Tr(X A U0 S) = Re Tr((X A) M0): one product X A per hit, which also is the
// new A when the hit is accepted (every warp takes the accept branch on almost
// every hit, so this halves the products per hit against carrying U and U S).
// The link is rebuilt as A U0 and reunitarised once after its hits.  The Markov
// chain is the one of U <- X U per accepted hit; only the rounding differs.
template <int ND, typename T, bool DF>
KLFT_D int site_update_exp(const Links<3, T> &U, const Geom &g, const Site &x, const MetroArgs &a, uint32_t sweep,
                           const Defect &df) {
  int nacc = 0;
  const ExpHitStream hs{(uint32_t)a.seed, (uint32_t)(a.seed >> 32) ^ (uint32_t)a.chain, site_lex(g, x), sweep};
  const long long lx = site_lin(g, x);
  const T bnc = (T)a.beta / T(3);
  const T half_eps = (T)(0.5 * a.eps);
#pragma unroll 1
  for (int mu = 0; mu < ND; ++mu) {
    if (open_link(g, x, mu)) continue;
    const uint32_t h0 = (uint32_t)(mu * a.nhits);
    // M0 = U0 S stays fixed; A is the product of the accepted X, so the current
    // link is A U0 and Re Tr(X A U0 S) = Re Tr((X A) M0): one product X A per hit
    const Mat<3, T> M0 = mul(U.load(lx, mu), staple<3, ND, T, DF>(U, g, x, mu, df));
    Mat<3, T> A = mident<3, T>();
    const bool dlink = DF && df.active && in_defect(g, df, x, mu);
    T trO = retr_diag(M0);
    bool changed = false;
    uint32_t aw[4];
    // the Philox words of hit h + 1 are drawn while hit h is evaluated
    uint32_t wn[8];
    hs.block(2 * h0, wn);
    hs.block(2 * h0 + 1, wn + 4);
#pragma unroll 1
    for (int hit = 0; hit < a.nhits; ++hit) {
      const uint32_t h = h0 + (uint32_t)hit;
      if (hit == 0 || (h & 3u) == 0u) hs.accept_block(h, aw);
      uint32_t w[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) w[k] = wn[k];
      if (hit + 1 < a.nhits) {
        hs.block(2 * (h + 1), wn);
        hs.block(2 * (h + 1) + 1, wn + 4);
      }
      const Mat<3, T> X = exp_proposal_w<T>(w, half_eps);
      const Mat<3, T> Y = hit == 0 ? X : mul(X, A);  // A is the identity before the first hit
      const T tY = retr_mul(Y, M0);
      T dS = -bnc * (tY - trO);
      if (dlink) dS *= (T)defect_c(df);
      const bool accept = dS < T(0) || accept_word(aw, h) < (double)exp(-dS);
      if (accept) {
        A = Y;
        trO = tY;
        ++nacc;
        changed = true;
      }
    }
    if (changed) U.store(lx, mu, restore(mul(A, U.load(lx, mu))));
  }
  return nacc;
}

}  // namespace klft
