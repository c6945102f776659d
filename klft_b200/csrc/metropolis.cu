// metropolis.cu -- one pass of the Metropolis sweep on one lattice.
//
// Reference proposals: sweep_Metropolis (Metropolis.hpp:118-178) visits the
// 2^Nd parity classes in the reference's order (class val has parity bit
// (val >> (Nd-1-d)) & 1 in dimension d, IndexHelper.hpp:84-93); the host
// enqueues one launch per class.  Sites of one class share no staple link, so
// a pass is race free.  exp(i eps H) proposals: 2 Nd link passes (mu, parity)
// of one thread per link (metropolis_site.cuh).  The per-site and per-link
// updates are in metropolis_site.cuh.
#include "metropolis_site.cuh"

namespace klft {

template <int NC, int ND, typename T, bool DF>
__global__ void __launch_bounds__(128, MinBlocks<T>::v)
    metropolis_ref_kernel(Links<NC, T> U, Geom g, int val, MetroArgs a, const uint32_t *__restrict__ d_sweep,
                          unsigned long long *__restrict__ d_nacc, Defect df) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int nacc = 0;
  if (t < g.Vh) nacc = site_update_ref<NC, ND, T, DF>(U, g, pass_site(g, t, val, ND), a, *d_sweep, df);
  add_accepts(nacc, d_nacc);
}

// link pass val = 2 MU + p: U_MU(x) of the V/2 sites of parity p (one
// instance per direction, so the staple's site steps are compiled)
template <int ND, typename T, bool DF, int MU>
__global__ void __launch_bounds__(128, MinBlocks<T>::v)
    metropolis_exp_kernel(Links<3, T> U, Geom g, int val, MetroArgs a, const uint32_t *__restrict__ d_sweep,
                          unsigned long long *__restrict__ d_nacc, Defect df) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int nacc = 0;
  bool ok = false;
  const Site x = link_pass_site(g, t, val & 1, ND, ok);
  if (ok && t < link_pass_threads(g, ND)) nacc = link_update_exp<ND, T, DF, MU>(U, g, x, MU, a, *d_sweep, df);
  add_accepts(nacc, d_nacc);
}

template <int NC, int ND, typename T, bool DF>
static cudaError_t launch_tdf(const Links<NC, T> &U, const Geom &g, int val, const MetroArgs &a,
                              const uint32_t *d_sweep, unsigned long long *d_nacc, const Defect &df, int block,
                              cudaStream_t st) {
  const unsigned grid = (unsigned)((g.Vh + block - 1) / block);
  if constexpr (NC == 3) {
    if (a.proposal == PROPOSAL_EXP) {
      const unsigned lgrid = (unsigned)((link_pass_threads(g, ND) + block - 1) / block);
      switch (val >> 1) {
        case 0: metropolis_exp_kernel<ND, T, DF, 0><<<lgrid, block, 0, st>>>(U, g, val, a, d_sweep, d_nacc, df); break;
        case 1: metropolis_exp_kernel<ND, T, DF, 1><<<lgrid, block, 0, st>>>(U, g, val, a, d_sweep, d_nacc, df); break;
        case 2:
          if constexpr (ND > 2)
            metropolis_exp_kernel<ND, T, DF, (ND > 2 ? 2 : 0)><<<lgrid, block, 0, st>>>(U, g, val, a, d_sweep, d_nacc,
                                                                                       df);
          break;
        default:
          if constexpr (ND > 3)
            metropolis_exp_kernel<ND, T, DF, (ND > 3 ? 3 : 0)><<<lgrid, block, 0, st>>>(U, g, val, a, d_sweep, d_nacc,
                                                                                       df);
          break;
      }
      return cudaGetLastError();
    }
  }
  metropolis_ref_kernel<NC, ND, T, DF><<<grid, block, 0, st>>>(U, g, val, a, d_sweep, d_nacc, df);
  return cudaGetLastError();
}

template <int NC, int ND, typename T>
static cudaError_t launch_t(void *links, const Geom &g, int val, const MetroArgs &a, const uint32_t *d_sweep,
                            unsigned long long *d_nacc, const Defect &df, int block, cudaStream_t st) {
  Links<NC, T> U{(cx<T> *)links, g.V};
  if (block != 32 && block != 64 && block != 128) block = 128;  // the kernels are built for <= 128 threads
  if (df.active) return launch_tdf<NC, ND, T, true>(U, g, val, a, d_sweep, d_nacc, df, block, st);
  return launch_tdf<NC, ND, T, false>(U, g, val, a, d_sweep, d_nacc, df, block, st);
}

template <int NC, typename T>
static cudaError_t launch_nd(int nd, void *links, const Geom &g, int val, const MetroArgs &a,
                             const uint32_t *d_sweep, unsigned long long *d_nacc, const Defect &df, int block,
                             cudaStream_t st) {
  switch (nd) {
    case 2: return launch_t<NC, 2, T>(links, g, val, a, d_sweep, d_nacc, df, block, st);
    case 3: return launch_t<NC, 3, T>(links, g, val, a, d_sweep, d_nacc, df, block, st);
    case 4: return launch_t<NC, 4, T>(links, g, val, a, d_sweep, d_nacc, df, block, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_metropolis_pass(int nc, int dtype, void *links, const Geom &g, int val, const MetroArgs &a,
                                   const uint32_t *d_sweep, unsigned long long *d_nacc, const Defect &df, int block,
                                   cudaStream_t st) {
  if (dtype == 0) {
    if (nc == 3 && a.proposal == 1) {
      // the FP64 exp(i eps H) proposal reads its Gaussians from the host-built table
      MetroArgs b = a;
      if (!(b.bm = bm_table())) return cudaErrorMemoryAllocation;
      return launch_nd<3, double>(g.nd, links, g, val, b, d_sweep, d_nacc, df, block, st);
    }
    switch (nc) {
      case 1: return launch_nd<1, double>(g.nd, links, g, val, a, d_sweep, d_nacc, df, block, st);
      case 2: return launch_nd<2, double>(g.nd, links, g, val, a, d_sweep, d_nacc, df, block, st);
      case 3: return launch_nd<3, double>(g.nd, links, g, val, a, d_sweep, d_nacc, df, block, st);
    }
  } else {
    switch (nc) {
      case 1: return launch_nd<1, float>(g.nd, links, g, val, a, d_sweep, d_nacc, df, block, st);
      case 2: return launch_nd<2, float>(g.nd, links, g, val, a, d_sweep, d_nacc, df, block, st);
      case 3: return launch_nd<3, float>(g.nd, links, g, val, a, d_sweep, d_nacc, df, block, st);
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
