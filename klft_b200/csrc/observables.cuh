// observables.cuh -- lattice-sum building blocks shared by the single-lattice
// observables (observables.cu) and the multi-chain batch kernels (batch.cu).
#pragma once
#include "common.cuh"

namespace klft {

constexpr int RED_THREADS = 256;

template <int THREADS>
KLFT_D double block_sum(double v) {
  __shared__ double red[THREADS / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < THREADS / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

// Site order for lattice-wide reductions: warp w takes parity class w mod 2^Nd
// and half-lattice sites [32 (w >> Nd), +32), so consecutive warps sweep all
// classes of one window of half-lattice sites and the neighbour links a warp
// needs were just brought into L2 by its sibling warps.  Coalescing is kept
// (a warp reads 32 consecutive entries of one class).
KLFT_D bool window_site(const Geom &g, long long t, Site &x, long long &lin) {
  // 2^Nd classes: shifts and masks; the half-coordinates in 32-bit arithmetic
  // whenever the half-volume allows (a 64-bit division by a run-time extent
  // costs tens of instructions)
  const long long w = t >> 5;
  const int sub = (int)(w & ((1 << g.nd) - 1));
  const long long hidx = (w >> g.nd) * 32 + (t & 31);
  if (hidx >= g.Vh) return false;
  if (g.Vh < (1LL << 31)) {
    unsigned r = (unsigned)hidx;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      const unsigned hd = (unsigned)g.H[d], q = r / hd;
      x.set_b(d, (sub >> d) & 1);
      x.set_h(d, (int)(r - q * hd));
      r = q;
    }
  } else {
    long long r = hidx;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      x.set_b(d, (sub >> d) & 1);
      x.set_h(d, (int)(r % g.H[d]));
      r /= g.H[d];
    }
  }
  lin = (long long)sub * g.Vh + hidx;
  return true;
}

KLFT_HD long long window_threads(const Geom &g) { return (long long)(1 << g.nd) * ((g.Vh + 31) / 32) * 32; }

template <typename T> struct PlaqMinBlocks { static constexpr int v = 2; };
template <> struct PlaqMinBlocks<double> { static constexpr int v = 1; };

// One block's share of the plaquette sum over the planes (mu, nu) with
// mu < nu < nu_end (nu_end = Nd: all planes): block b of nb over the window
// order (the partial that plaquette_kernel's block b writes).
// F64 = true sums every product term in FP64 (the HMC action, whose differences
// decide acceptance); otherwise each plane's trace is formed in the link
// precision and the lattice sum in FP64.
template <int NC, int ND, typename T, bool F64 = false>
KLFT_D double plaquette_partial(const Links<NC, T> &U, const Geom &g, int nu_end, long long b, long long nb) {
  double acc = 0.0;
  const long long nthr = window_threads(g);
  for (long long t = b * RED_THREADS + threadIdx.x; t < nthr; t += nb * RED_THREADS) {
    Site x;
    long long lin;
    if (!window_site(g, t, x, lin)) continue;
    // unrolled over (mu, nu): the site steps fold to a few integer operations
#pragma unroll
    for (int mu = 0; mu < ND; ++mu) {
      const Site xpmu = site_up(g, x, mu);
      const Mat<NC, T> umu = U.load(lin, mu);
#pragma unroll
      for (int nu = mu + 1; nu < ND; ++nu) {
        if (nu >= nu_end) break;
        const Mat<NC, T> lmu = mul(umu, U.load(site_lin(g, xpmu), nu));
        const Mat<NC, T> lnu = mul(U.load(lin, nu), U.load(site_lin(g, site_up(g, x, nu)), mu));
        if constexpr (F64) acc += retr_nd<NC, T, double>(lmu, lnu);
        else acc += (double)retr_nd<NC, T, T>(lmu, lnu);
      }
    }
  }
  return acc;
}

}  // namespace klft
