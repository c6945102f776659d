// metropolis_site.cuh -- the Metropolis updates shared by the single-lattice
// pass kernels (metropolis.cu) and the multi-chain batch kernels (batch.cu).
//
// Semantics follow MetropolisGaugeField::operator() (Metropolis.hpp:73-113):
// per link the staple is formed once, then nHits proposals are accepted with
// probability min(1, exp(-dS)), dS = -(beta/Nc) Re Tr[(U' - U) S], and an
// accepted link is stored reunitarised (restoreSUN).  With the reference
// proposals (U' = U r) a thread owns one site of a parity class and updates its
// Nd links in order mu = 0..Nd-1, the reference's order (site_update_ref).  The
// SU(3) exp(i eps H) proposal (U' = X U, no reference counterpart) runs one
// thread per link in 2 Nd link passes (link_update_exp).
//
// Per-hit cost: with M = S U, Re Tr(U r S) = Re Tr(r M) needs only the diagonal
// of r M.  SU(3) reference proposals (a few per cent accepted) rebuild U r and M
// on acceptance; U(1)/SU(2) and the exp(i eps H) proposals, accepted on
// ~30-70 % of hits (so every warp runs the accept branch on nearly every hit),
// accumulate the accepted proposals into one matrix A instead and need one
// product per hit.
//
// Random numbers: the reference proposals (U(1), SU(2), the SU(3)
// Gram-Schmidt generator) consume the site's sequential Philox stream in the
// order the reference functor consumes its generator.  The exp(i eps H)
// proposal (expprop.cuh) reads fixed stream positions per hit, so a proposal
// does not depend on earlier accept decisions.  Neither depends on the launch
// shape.
#pragma once
#include "expprop.cuh"
#include "group.cuh"
#include "kernels.cuh"
#include "staple.cuh"

namespace klft {

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
// The hits of link U_mu(x) in the reference's order (Metropolis.hpp:85-107),
// drawing from the site's stream rng.  MU >= 0: mu at compile time (the staple's
// site steps compiled, its nu loops unrolled); MU = -1: run-time mu.
template <int NC, int ND, typename T, bool DF, int MU>
KLFT_D int link_update_ref(const Links<NC, T> &U, const Geom &g, const Site &x, int mu, const MetroArgs &a,
                           const Defect &df, Stream &rng, long long lx, T bnc) {
  if (open_link(g, x, mu)) return 0;
  int nacc = 0;
  Mat<NC, T> S;
  if constexpr (MU >= 0) S = staple_ct<NC, ND, (MU >= 0 ? MU : 0), T>(U, g, x);
  else S = staple<NC, ND, T, DF>(U, g, x, mu, df);
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
    return nacc;
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
  return nacc;
}

template <int NC, int ND, typename T, bool DF>
KLFT_D int site_update_ref(const Links<NC, T> &U, const Geom &g, const Site &x, const MetroArgs &a, uint32_t sweep,
                           const Defect &df) {
  int nacc = 0;
  Stream rng(a.seed, a.chain, site_lex(g, x), sweep, KIND_METROPOLIS, 0);
  const long long lx = site_lin(g, x);
  const T bnc = (T)a.beta / (T)NC;
  if constexpr (NC <= 2 && !DF) {
    // U(1), SU(2): the directions unrolled, each with its compiled staple
    nacc += link_update_ref<NC, ND, T, DF, 0>(U, g, x, 0, a, df, rng, lx, bnc);
    nacc += link_update_ref<NC, ND, T, DF, 1>(U, g, x, 1, a, df, rng, lx, bnc);
    if constexpr (ND > 2) nacc += link_update_ref<NC, ND, T, DF, (ND > 2 ? 2 : 0)>(U, g, x, 2, a, df, rng, lx, bnc);
    if constexpr (ND > 3) nacc += link_update_ref<NC, ND, T, DF, (ND > 3 ? 3 : 0)>(U, g, x, 3, a, df, rng, lx, bnc);
  } else {
#pragma unroll 1
    for (int mu = 0; mu < ND; ++mu) nacc += link_update_ref<NC, ND, T, DF, -1>(U, g, x, mu, a, df, rng, lx, bnc);
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
//
// The exp proposal has no reference chain to follow, so its sweep visits the
// links in 2 Nd "link passes" (mu, p) instead of the reference's 2^Nd site
// classes: pass (mu, p) updates U_mu(x) for every site x of parity
// p = sum_d x_d mod 2.  The staple of U_mu(x) reads U_mu only at x +- nu (the
// other parity) and U_nu, nu != mu, which the pass does not change, so the
// links of a pass are independent.  A pass is V/2 threads, one link each
// (the reference-proposal update keeps one thread per site of a class and the
// reference's order, for hit-by-hit parity with klft).

// Site t of the sites of parity p.  Within a pass the threads run over chunks
// of 32 consecutive half-lattice indices hidx, and within a chunk over the
// 2^(Nd-1) site classes of that parity (class c: bits sub = (c << 1) | b0, b0
// fixing the parity): a warp reads 32 consecutive sites of one class
// (coalesced), and the warps in flight at any time share one small hidx window,
// so the staple neighbourhoods they read are reused from L2.  Threads
// t < link_pass_threads(g, nd) cover the V/2 sites once; those with hidx >= Vh
// (Vh not a multiple of 32) have no site (ok = false).
KLFT_HD long long link_pass_threads(const Geom &g, int nd) {
  return (g.Vh + 31) / 32 * 32 * (1ll << (nd - 1));
}
KLFT_D Site link_pass_site(const Geom &g, long long t, int p, int nd, bool &ok) {
  const unsigned lane = (unsigned)(t & 31);
  const unsigned long long w = (unsigned long long)(t >> 5);
  const unsigned c = (unsigned)(w & ((1u << (nd - 1)) - 1u));  // 2^(Nd-1) classes per parity
  unsigned hidx = (unsigned)((w >> (nd - 1)) * 32u + lane);
  ok = hidx < (unsigned)g.Vh;
  const unsigned sub = (c << 1) | ((unsigned)(__popc(c) & 1) ^ (unsigned)p);
  Site x;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    x.set_b(d, d < nd ? (int)((sub >> d) & 1u) : 0);
    const unsigned hd = (unsigned)g.H[d];
    const unsigned q = hidx / hd;
    x.set_h(d, (int)(hidx - q * hd));
    hidx = q;
  }
  return x;
}

// One hit: Y = X A (A is the identity before the first hit), the action
// change against the current Re Tr(A M0) = trO, the accept test with the hit's
// FP64 uniform; on acceptance A <- Y.
template <typename T>
KLFT_D void exp_hit(const Mat<3, T> &X, bool first, const Mat<3, T> &M0, T bnc, T cdef, const uint32_t aw[4],
                    uint32_t h, Mat<3, T> &A, T &trO, int &nacc) {
  const Mat<3, T> Y = first ? X : mul(X, A);
  const T tY = retr_mul(Y, M0);
  const T dS = -bnc * (tY - trO) * cdef;
  const bool accept = dS < T(0) || accept_word(aw, h) < (double)exp(-dS);
  if (accept) {
    A = Y;
    trO = tY;
    ++nacc;
  }
}

// The hits of link U_mu(x) (hit h = mu * nHits + hit of the site's stream).
// MU: the pass's direction at compile time (mu == MU; every link pass, single
// lattice or batch, is one kernel instance per direction), for the staples
// with compiled site steps.
template <int ND, typename T, bool DF, int MU>
KLFT_D int link_update_exp(const Links<3, T> &U, const Geom &g, const Site &x, int mu, const MetroArgs &a,
                           uint32_t sweep, const Defect &df) {
  static_assert(MU >= 0 && MU < ND, "link passes are compiled per direction");
  if (open_link(g, x, mu)) return 0;
  int nacc = 0;
  const ExpHitStream hs{(uint32_t)a.seed, (uint32_t)(a.seed >> 32) ^ (uint32_t)a.chain, site_lex(g, x), sweep, a.bm};
  const long long lx = site_lin(g, x);
  const T bnc = (T)a.beta / T(3);
  const T half_eps = (T)(0.5 * a.eps);
  const uint32_t h0 = (uint32_t)(mu * a.nhits);
  const T cdef = DF && df.active && in_defect(g, df, x, mu) ? (T)defect_c(df) : T(1);
  // M0 = U0 S stays fixed; A is the product of the accepted X, so the current
  // link is A U0 and Re Tr(X A U0 S) = Re Tr((X A) M0): one product X A per hit
  Mat<3, T> S;
  if constexpr (!DF && sizeof(T) == 4) S = staple_su3_2row_ct<ND, MU>(U, g, x);
  else S = staple_ct<3, ND, MU, T, DF>(U, g, x, df);
  const Mat<3, T> M0 = mul(U.load(lx, mu), S);
  Mat<3, T> A = mident<3, T>();
  T trO = retr_diag(M0);
  uint32_t aw[4];
#pragma unroll 1
  for (int hit = 0; hit < a.nhits; ++hit) {
    const uint32_t h = h0 + (uint32_t)hit;
    if (hit == 0 || (h & 3u) == 0u) hs.accept_block(h, aw);
    exp_hit<T>(exp_proposal<T>(hs, h, half_eps), hit == 0, M0, bnc, cdef, aw, h, A, trO, nacc);
  }
  if (nacc) U.store(lx, mu, restore(mul(A, U.load(lx, mu))));
  return nacc;
}

}  // namespace klft
