// observables.cu -- gauge observables as single fused launches with FP64
// accumulation and an ordered (deterministic) two-stage reduction.
//
// GaugePlaquette (GaugePlaquette.hpp:36-135): per site the sum over mu < nu of
//   Re Tr[(U_mu(x) U_nu(x+mu)) (U_nu(x) U_mu(x+nu))^+],
// reduced over the lattice in one kernel (the reference writes a per-site field
// and reduces it in a second pass).
//
// Wilson loops, direct form (WilsonLoop.hpp:34-245): for each (Lmu, Lnu) pair
//   Re Tr[(WLmu(x) WLnu(x+Lmu mu)) (WLnu(x) WLmu(x+Lnu nu))^+]
// with lines built by right-multiplication.  Kept as the simple cross-check
// form of the gauge-fixed kernel in wilson.cu.
#include "common.cuh"
#include "kernels.cuh"
#include "observables.cuh"

namespace klft {

template <int NC, int ND, typename T, bool F64>
__global__ void __launch_bounds__(RED_THREADS, PlaqMinBlocks<T>::v) plaquette_kernel(Links<NC, T> U, Geom g,
                                                                                     double *part, int nu_end) {
  const double s =
      block_sum<RED_THREADS>(plaquette_partial<NC, ND, T, F64>(U, g, nu_end, blockIdx.x, gridDim.x));
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

template <int NC, typename T>
KLFT_D Mat<NC, T> wline(const Links<NC, T> &U, const Geom &g, Site s, int d, int len) {
  Mat<NC, T> l = U.load(site_lin(g, s), d);
  for (int i = 1; i < len; ++i) {
    s = site_up(g, s, d);
    l = mul(l, U.load(site_lin(g, s), d));
  }
  return l;
}

template <int NC, typename T>
__global__ void __launch_bounds__(RED_THREADS) wilson_direct_kernel(Links<NC, T> U, Geom g, int mu, int nu,
                                                                    const int *pairs, int npairs, double *part) {
  for (int k = 0; k < npairs; ++k) {
    const int Lmu = pairs[2 * k], Lnu = pairs[2 * k + 1];
    double acc = 0.0;
    for (long long lin = (long long)blockIdx.x * RED_THREADS + threadIdx.x; lin < g.V;
         lin += (long long)gridDim.x * RED_THREADS) {
      const Site x = site_from_lin(g, lin);
      Mat<NC, T> lmu, lnu;
      if (Lmu == 0 && Lnu == 0) {
        lmu = mident<NC, T>();
        lnu = mident<NC, T>();
      } else if (Lmu == 0) {
        lmu = wline(U, g, x, nu, Lnu);
        lnu = lmu;
      } else if (Lnu == 0) {
        lmu = wline(U, g, x, mu, Lmu);
        lnu = lmu;
      } else {
        lmu = mul(wline(U, g, x, mu, Lmu), wline(U, g, site_shift(g, x, mu, Lmu), nu, Lnu));
        lnu = mul(wline(U, g, x, nu, Lnu), wline(U, g, site_shift(g, x, nu, Lnu), mu, Lmu));
      }
      acc += retr_nd<NC, T, double>(lmu, lnu);
    }
    const double s = block_sum<RED_THREADS>(acc);
    if (threadIdx.x == 0) part[(long long)k * gridDim.x + blockIdx.x] = s;
  }
}

// out[k] = sum_i part[k * nblk + i], one block per output, fixed order
__global__ void reduce_partials_kernel(const double *part, int nblk, double *out) {
  const int k = blockIdx.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < nblk; i += RED_THREADS) v += part[(long long)k * nblk + i];
  const double s = block_sum<RED_THREADS>(v);
  if (threadIdx.x == 0) out[k] = s;
}

int plaquette_blocks(const Geom &g) {
  long long nb = (g.V + RED_THREADS - 1) / RED_THREADS;
  return (int)(nb < 148 * 8 ? nb : 148 * 8);
}

cudaError_t launch_reduce_partials(const double *d_part, int nblk, int n, double *d_out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  reduce_partials_kernel<<<n, RED_THREADS, 0, st>>>(d_part, nblk, d_out);
  return cudaGetLastError();
}

#define KLFT_OBS_DISPATCH(nc, dtype, nd, KERNEL_CALL)                           \
  do {                                                                         \
    if (dtype == 0) {                                                          \
      using T = double;                                                        \
      if (nc == 1) { constexpr int NC = 1; KERNEL_CALL; }                      \
      else if (nc == 2) { constexpr int NC = 2; KERNEL_CALL; }                 \
      else if (nc == 3) { constexpr int NC = 3; KERNEL_CALL; }                 \
      else return cudaErrorInvalidValue;                                       \
    } else {                                                                   \
      using T = float;                                                         \
      if (nc == 1) { constexpr int NC = 1; KERNEL_CALL; }                      \
      else if (nc == 2) { constexpr int NC = 2; KERNEL_CALL; }                 \
      else if (nc == 3) { constexpr int NC = 3; KERNEL_CALL; }                 \
      else return cudaErrorInvalidValue;                                       \
    }                                                                          \
  } while (0)

cudaError_t launch_plaquette(int nc, int dtype, const void *links, const Geom &g, double *d_part, int nblk,
                             double *d_out, cudaStream_t st, int nu_end, bool f64_terms) {
  if (nu_end < 0) nu_end = g.nd;
#define KLFT_PQ(NDV)                                                                                              \
  do {                                                                                                            \
    if (f64_terms)                                                                                                \
      plaquette_kernel<NC, NDV, T, true><<<nblk, RED_THREADS, 0, st>>>(Links<NC, T>{(cx<T> *)links, g.V}, g,      \
                                                                       d_part, nu_end);                           \
    else                                                                                                          \
      plaquette_kernel<NC, NDV, T, false><<<nblk, RED_THREADS, 0, st>>>(Links<NC, T>{(cx<T> *)links, g.V}, g,     \
                                                                        d_part, nu_end);                          \
  } while (0)
  KLFT_OBS_DISPATCH(nc, dtype, g.nd, ({
    if (g.nd == 2) KLFT_PQ(2);
    else if (g.nd == 3) KLFT_PQ(3);
    else KLFT_PQ(4);
  }));
#undef KLFT_PQ
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_reduce_partials(d_part, nblk, 1, d_out, st);
}

cudaError_t launch_wilson_direct(int nc, int dtype, const void *links, const Geom &g, int mu, int nu,
                                 const int *d_pairs, int npairs, double *d_part, int nblk, double *d_out,
                                 cudaStream_t st) {
  KLFT_OBS_DISPATCH(nc, dtype, g.nd, (wilson_direct_kernel<NC, T><<<nblk, RED_THREADS, 0, st>>>(
                                          Links<NC, T>{(cx<T> *)links, g.V}, g, mu, nu, d_pairs, npairs, d_part)));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_reduce_partials(d_part, nblk, npairs, d_out, st);
}

}  // namespace klft
