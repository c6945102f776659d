// metropolis.cu -- one parity-class pass of the Metropolis sweep.
//
// Semantics follow MetropolisGaugeField::operator() (Metropolis.hpp:73-113) and
// sweep_Metropolis (Metropolis.hpp:118-178): the sweep visits the 2^Nd parity
// classes in the reference's order (class val has parity bit
// (val >> (Nd-1-d)) & 1 in dimension d, IndexHelper.hpp:84-93); a thread owns
// one site of the class and updates its Nd links in order mu = 0..Nd-1; per
// link the staple is formed once, then nHits proposals U' = U r are accepted
// with probability min(1, exp(-dS)), dS = -(beta/Nc) Re Tr[(U' - U) S], and an
// accepted link is stored reunitarised (restoreSUN).  Sites of one class share
// no staple link, so the pass is race free.
//
// Per-hit cost is cut by carrying M = S U: Re Tr(U r S) = Re Tr(r M) needs only
// the diagonal of r M (36 flops for SU(3)) instead of the product U r; U r and M
// are rebuilt only on acceptance.  The random numbers come from the site's own
// Philox stream (key = seed/chain, counter = sweep/site), consumed in the same
// order as the reference functor consumes its generator, so the result does not
// depend on the launch shape.
#include "group.cuh"
#include "kernels.cuh"
#include "staple.cuh"

namespace klft {

template <int NC, int ND, typename T>
__global__ void __launch_bounds__(128) metropolis_pass_kernel(Links<NC, T> U, Geom g, int val, MetroArgs a,
                                                              const uint32_t *__restrict__ d_sweep,
                                                              unsigned long long *__restrict__ d_nacc, Defect df) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int nacc = 0;
  if (t < g.Vh) {
    Site x;
    long long r = t;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      x.h[d] = (int)(r % g.H[d]);
      r /= g.H[d];
      x.b[d] = d < ND ? (val >> (ND - 1 - d)) & 1 : 0;
    }
    const uint32_t sweep = *d_sweep;
    Stream rng(a.seed, a.chain, site_lex(g, x), sweep, KIND_METROPOLIS, 0);
    const long long lx = site_lin(g, x);
    const T bnc = (T)a.beta / (T)NC;
#pragma unroll 1
    for (int mu = 0; mu < ND; ++mu) {
      const Mat<NC, T> S = staple<NC, ND, T>(U, g, x, mu, df);
      const bool dlink = df.active && in_defect(g, df, x, mu);
      const T c = dlink ? (T)df.c : T(1);
      Mat<NC, T> Uo = U.load(lx, mu);
      Mat<NC, T> M = mul(S, Uo);
      T trO = T(0);
#pragma unroll
      for (int i = 0; i < NC; ++i) trO += M.e[i][i].re;
      bool changed = false;
#pragma unroll 1
      for (int hit = 0; hit < a.nhits; ++hit) {
        const Mat<NC, T> rr = propose<T>(rng, (const Mat<NC, T> *)nullptr, a.delta, a.proposal, a.eps);
        const T trN = retr_mul(rr, M);
        T dS = -bnc * (trN - trO);
        if (dlink) dS *= c;
        bool accept = dS < T(0);
        if (!accept) accept = rng.next() < (double)exp(-dS);
        if (accept) {
          Uo = restore(mul(Uo, rr));
          M = mul(S, Uo);
          trO = T(0);
#pragma unroll
          for (int i = 0; i < NC; ++i) trO += M.e[i][i].re;
          ++nacc;
          changed = true;
        }
      }
      if (changed) U.store(lx, mu, Uo);
    }
  }
  // block total of accepted hits -> one atomic per block
  __shared__ int red[4];
  int v = warp_sum(nacc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    if (s) atomicAdd(d_nacc, (unsigned long long)s);
  }
}

template <int NC, int ND, typename T>
static cudaError_t launch_t(void *links, const Geom &g, int val, const MetroArgs &a, const uint32_t *d_sweep,
                            unsigned long long *d_nacc, const Defect &df, cudaStream_t st) {
  Links<NC, T> U{(cx<T> *)links, g.V};
  const int block = 128;
  const long long grid = (g.Vh + block - 1) / block;
  metropolis_pass_kernel<NC, ND, T><<<(unsigned)grid, block, 0, st>>>(U, g, val, a, d_sweep, d_nacc, df);
  return cudaGetLastError();
}

template <int NC, typename T>
static cudaError_t launch_nd(int nd, void *links, const Geom &g, int val, const MetroArgs &a,
                             const uint32_t *d_sweep, unsigned long long *d_nacc, const Defect &df, cudaStream_t st) {
  switch (nd) {
    case 2: return launch_t<NC, 2, T>(links, g, val, a, d_sweep, d_nacc, df, st);
    case 3: return launch_t<NC, 3, T>(links, g, val, a, d_sweep, d_nacc, df, st);
    case 4: return launch_t<NC, 4, T>(links, g, val, a, d_sweep, d_nacc, df, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_metropolis_pass(int nc, int dtype, void *links, const Geom &g, int val, const MetroArgs &a,
                                   const uint32_t *d_sweep, unsigned long long *d_nacc, const Defect &df, int,
                                   cudaStream_t st) {
  if (dtype == 0) {
    switch (nc) {
      case 1: return launch_nd<1, double>(g.nd, links, g, val, a, d_sweep, d_nacc, df, st);
      case 2: return launch_nd<2, double>(g.nd, links, g, val, a, d_sweep, d_nacc, df, st);
      case 3: return launch_nd<3, double>(g.nd, links, g, val, a, d_sweep, d_nacc, df, st);
    }
  } else {
    switch (nc) {
      case 1: return launch_nd<1, float>(g.nd, links, g, val, a, d_sweep, d_nacc, df, st);
      case 2: return launch_nd<2, float>(g.nd, links, g, val, a, d_sweep, d_nacc, df, st);
      case 3: return launch_nd<3, float>(g.nd, links, g, val, a, d_sweep, d_nacc, df, st);
    }
  }
  return cudaErrorInvalidValue;
}

__global__ void advance_kernel(uint32_t *c) { c[0] += 1u; }

cudaError_t launch_advance(uint32_t *d_counter, cudaStream_t st) {
  advance_kernel<<<1, 1, 0, st>>>(d_counter);
  return cudaGetLastError();
}

}  // namespace klft
