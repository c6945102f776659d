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
// proposal (no reference counterpart, expprop.cuh) reads fixed stream positions
// per hit, so a proposal does not depend on earlier accept decisions.  Neither
// depends on the launch shape.
#pragma once
#include <type_traits>

#include "expprop.cuh"
#include "group.cuh"
#include "kernels.cuh"
#include "staple.cuh"

#ifndef KLFT_EXP_PAIRS
#define KLFT_EXP_PAIRS 1
#endif
#ifndef KLFT_EXP_M0_SMEM
#define KLFT_EXP_M0_SMEM 1
#endif

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
//
// One hit: Y = X A (A is the identity before the first hit), the action
// change against the current Re Tr(A M0) = trO, the accept test with the hit's
// FP64 uniform; on acceptance A <- Y.
// Re Tr(Y M0) with M0 in shared memory (entry (k, i) at mq[(3 k + i) * 128])
KLFT_D float retr_mul_shared(const Mat<3, float> &Y, const float2 *mq) {
  float tY = 0.0f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float2 m0 = mq[(0 * 3 + i) * 128], m1 = mq[(1 * 3 + i) * 128], m2 = mq[(2 * 3 + i) * 128];
    float s = Y.e[i][0].re * m0.x - Y.e[i][0].im * m0.y;
    s = fmaf(Y.e[i][1].re, m1.x, s);
    s = fmaf(-Y.e[i][1].im, m1.y, s);
    s = fmaf(Y.e[i][2].re, m2.x, s);
    s = fmaf(-Y.e[i][2].im, m2.y, s);
    tY += s;
  }
  return tY;
}

template <typename T, typename MT>
KLFT_D void exp_hit(const Mat<3, T> &X, bool first, const MT &M0, T bnc, T cdef, const uint32_t aw[4],
                    uint32_t h, Mat<3, T> &A, T &trO, int &nacc) {
  const Mat<3, T> Y = first ? X : mul(X, A);
  T tY;
  if constexpr (std::is_same<MT, Mat<3, T>>::value) tY = retr_mul(Y, M0);
  else tY = retr_mul_shared(Y, M0);
  const T dS = -bnc * (tY - trO) * cdef;
  const bool accept = dS < T(0) || accept_word(aw, h) < (double)exp(-dS);
  if (accept) {
    A = Y;
    trO = tY;
    ++nacc;
  }
}

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
    const T cdef = DF && df.active && in_defect(g, df, x, mu) ? (T)defect_c(df) : T(1);
    T trO = retr_diag(M0);
    const int nacc0 = nacc;
    uint32_t aw[4];
    if constexpr (sizeof(T) == 4 && KLFT_EXP_PAIRS) {
      // FP32: the proposals of hits h and h + 1 are built together, one hit in
      // each lane of packed FP32 pairs, then evaluated in turn; the second one
      // waits in shared memory (one 8-byte complex per entry and thread, so a
      // warp's accesses are 256 contiguous bytes) while the first is evaluated
      __shared__ float2 xs[9][128];
      float2 *xq = &xs[0][threadIdx.x];
#if KLFT_EXP_M0_SMEM
      __shared__ float2 ms[9][128];
      float2 *mq = &ms[0][threadIdx.x];
#pragma unroll
      for (int k = 0; k < 9; ++k) mq[k * 128] = make_float2(M0.e[k / 3][k % 3].re, M0.e[k / 3][k % 3].im);
#endif
#pragma unroll 1
      for (int hit = 0; hit < a.nhits; hit += 2) {
        const uint32_t h = h0 + (uint32_t)hit;
        const bool two = hit + 1 < a.nhits;
        Mat<3, T> X;
        {
          const XMat<float2> P = exp_proposal_pair(hs, h, half_eps, two);
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              X.e[i][j] = mk<T>(P.re[i][j].x, P.im[i][j].x);
              xq[(i * 3 + j) * 128] = make_float2(P.re[i][j].y, P.im[i][j].y);
            }
        }
        if (hit == 0 || (h & 3u) == 0u) hs.accept_block(h, aw);
#if KLFT_EXP_M0_SMEM
        exp_hit<T>(X, hit == 0, (const float2 *)mq, bnc, cdef, aw, h, A, trO, nacc);
#else
        exp_hit<T>(X, hit == 0, M0, bnc, cdef, aw, h, A, trO, nacc);
#endif
        if (two) {
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              const float2 v = xq[(i * 3 + j) * 128];
              X.e[i][j] = mk<T>(v.x, v.y);
            }
          if (((h + 1u) & 3u) == 0u) hs.accept_block(h + 1u, aw);
#if KLFT_EXP_M0_SMEM
          exp_hit<T>(X, false, (const float2 *)mq, bnc, cdef, aw, h + 1u, A, trO, nacc);
#else
          exp_hit<T>(X, false, M0, bnc, cdef, aw, h + 1u, A, trO, nacc);
#endif
        }
      }
    } else {
#pragma unroll 1
      for (int hit = 0; hit < a.nhits; ++hit) {
        const uint32_t h = h0 + (uint32_t)hit;
        if (hit == 0 || (h & 3u) == 0u) hs.accept_block(h, aw);
        exp_hit<T>(exp_proposal<T>(hs, h, half_eps), hit == 0, M0, bnc, cdef, aw, h, A, trO, nacc);
      }
    }
    if (nacc != nacc0) U.store(lx, mu, restore(mul(A, U.load(lx, mu))));
  }
  return nacc;
}

}  // namespace klft
