// diag.cu -- diagnostics with no counterpart in the reference:
//  * measured CUDA-core peaks used as roofline denominators for the kernels of
//    this library (they run on the FP32/FP64 pipes, not tensor cores): a grid of
//    independent FMA chains, long enough to amortise launch overhead;
//  * the error of the mixed form's Metropolis action change against FP64 on one
//    configuration, hit by hit with identical proposals.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/klft_b200.h"
#include "capi_internal.h"
#include "metropolis_site.cuh"

namespace klft {

template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T *out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x, x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3), x4 = x0 + T(4), x5 = x0 + T(5),
    x6 = x0 + T(6), x7 = x0 + T(7);
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-12345.678)) out[0] = s;  // keeps the chains alive
}

// FP64 link -> the mixed form's stored link (two FP32 rows, third row rebuilt
// in FP32 as conj(row0 x row1)), promoted back to FP64 for the FP32 products
KLFT_D Mat<3, float> to_mixed(const Mat<3, double> &u) {
  Mat<3, float> m;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.e[i][j] = mk<float>((float)u.e[i][j].re, (float)u.e[i][j].im);
  m.e[2][0] = conj(m.e[0][1] * m.e[1][2] - m.e[0][2] * m.e[1][1]);
  m.e[2][1] = conj(m.e[0][2] * m.e[1][0] - m.e[0][0] * m.e[1][2]);
  m.e[2][2] = conj(m.e[0][0] * m.e[1][1] - m.e[0][1] * m.e[1][0]);
  return m;
}

// Per link of an FP64 SU(3) lattice and per hit of the exp(i eps H) stream of
// sweep `sweep`: dS64 from the FP64 links and FP64 arithmetic, dS32 from the
// links as the mixed form stores them and FP32 arithmetic (the first-hit form
// -beta/3 Re Tr((X - 1) U S), with the same X drawn in each precision), and
// whether the hit's accept uniform decides differently.  Sums per block into
// acc: [n, sum d, sum d^2, sum dS64 d, sum dS64^2, flips], d = dS32 - dS64; the
// largest |d| as the bits of a non-negative double.
__global__ void __launch_bounds__(128) dS_error_kernel(Links<3, double> U, Geom g, double beta, double eps, int nhits,
                                                       uint64_t seed, uint64_t chain, uint32_t sweep, double *acc,
                                                       unsigned long long *dmax, const double *bm) {
  const long long lin = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double loc[6] = {0, 0, 0, 0, 0, 0};
  double m = 0.0;
  if (lin < g.V) {
    const Site x = site_from_lin(g, lin);
    const ExpHitStream hs{(uint32_t)seed, (uint32_t)(seed >> 32) ^ (uint32_t)chain, site_lex(g, x), sweep, bm};
    for (int mu = 0; mu < g.nd; ++mu) {
      // staple in FP64, and in FP32 from the mixed form's links
      Mat<3, double> S64 = mzero<3, double>();
      Mat<3, float> S32 = mzero<3, float>();
      const Site xpmu = site_up(g, x, mu);
      for (int nu = 0; nu < g.nd; ++nu) {
        if (nu == mu) continue;
        const Site xpnu = site_up(g, x, nu), xpmu_mnu = site_dn(g, xpmu, nu), xmnu = site_dn(g, x, nu);
        const Mat<3, double> a = U.load(site_lin(g, xpmu), nu), b = U.load(site_lin(g, xpnu), mu),
                             c = U.load(site_lin(g, x), nu), d = U.load(site_lin(g, xpmu_mnu), nu),
                             e = U.load(site_lin(g, xmnu), mu), f = U.load(site_lin(g, xmnu), nu);
        madd(S64, mul_nd(mul_nd(a, b), c));
        madd(S64, mul(mul_dd(d, e), f));
        madd(S32, mul_nd(mul_nd(to_mixed(a), to_mixed(b)), to_mixed(c)));
        madd(S32, mul(mul_dd(to_mixed(d), to_mixed(e)), to_mixed(f)));
      }
      const Mat<3, double> u = U.load(lin, mu);
      const Mat<3, double> M64 = mul(u, S64);
      const Mat<3, float> M32 = mul(to_mixed(u), S32);
      const double tr64 = retr_diag(M64);
      const float tr32 = retr_diag(M32);
      uint32_t aw[4];
      for (int hit = 0; hit < nhits; ++hit) {
        const uint32_t h = (uint32_t)(mu * nhits + hit);
        if (hit == 0 || (h & 3u) == 0u) hs.accept_block(h, aw);
        const double dS64 = -(beta / 3.0) * (retr_mul(exp_proposal<double>(hs, h, 0.5 * eps), M64) - tr64);
        const float dS32 = -((float)beta / 3.0f) * (retr_mul(exp_proposal<float>(hs, h, (float)(0.5 * eps)), M32) - tr32);
        const double d = (double)dS32 - dS64;
        const double uacc = accept_word(aw, h);
        const bool a64 = dS64 < 0.0 || uacc < exp(-dS64);
        const bool a32 = dS32 < 0.0f || uacc < (double)expf(-dS32);
        loc[0] += 1.0;
        loc[1] += d;
        loc[2] += d * d;
        loc[3] += dS64 * d;
        loc[4] += dS64 * dS64;
        loc[5] += a64 != a32 ? 1.0 : 0.0;
        m = fmax(m, fabs(d));
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double v = warp_sum(loc[k]);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&acc[k], v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(dmax, (unsigned long long)__double_as_longlong(m));
}

}  // namespace klft

using namespace klft;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

extern "C" klft_status klft_exp_proposal_dS_error(klft_lattice *lat, double beta, double eps, int nhits,
                                                  double *out) {
  if (!lat || !out) return fail(KLFT_EINVAL, "klft_exp_proposal_dS_error: null pointer");
  if (lat->nc != 3 || lat->precision != KLFT_PRECISION_FP64)
    return fail(KLFT_EINVAL, "klft_exp_proposal_dS_error: needs an FP64 SU(3) lattice");
  if (nhits < 1 || !(eps == eps)) return fail(KLFT_EINVAL, "klft_exp_proposal_dS_error: bad nhits or eps");
  std::lock_guard<std::mutex> guard(lat->mtx);
  CK(lat->s_aux.ensure(8 * sizeof(double)));
  double *d_acc = (double *)lat->s_aux.ptr;
  CK(cudaMemsetAsync(d_acc, 0, 8 * sizeof(double), lat->stream));
  uint32_t sweep = 0;
  CK(cudaMemcpyAsync(&sweep, lat->d_counters, sizeof sweep, cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  const double *bm = bm_table();
  if (!bm) return fail(KLFT_ECUDA, "klft_exp_proposal_dS_error: Box-Muller table unavailable");
  const unsigned grid = (unsigned)((lat->g.V + 127) / 128);
  dS_error_kernel<<<grid, 128, 0, lat->stream>>>(Links<3, double>{(cx<double> *)lat->links, lat->g.V}, lat->g, beta,
                                                 eps, nhits, lat->seed, lat->chain, sweep, d_acc,
                                                 (unsigned long long *)(d_acc + 6), bm);
  CK(cudaGetLastError());
  double h[8];
  CK(cudaMemcpyAsync(h, d_acc, sizeof h, cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  const double n = h[0];
  out[0] = n;
  out[1] = h[1] / n;                                              // mean d
  out[2] = sqrt(h[2] / n);                                        // rms d
  unsigned long long bits;
  memcpy(&bits, &h[6], sizeof bits);
  out[3] = __builtin_bit_cast(double, bits);                      // max |d|
  out[4] = h[4] > 0.0 ? h[3] / h[4] : 0.0;                        // slope of d against dS64
  out[5] = h[5] / n;                                              // fraction of hits decided differently
  return KLFT_OK;
}

extern "C" klft_status klft_peak_flops(int dtype, double *tflops) {
  if (!tflops) return fail(KLFT_EINVAL, "klft_peak_flops: null pointer");
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "klft_peak_flops");
  void *buf = nullptr;
  if ((e = cudaMalloc(&buf, 64)) != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  const int blocks = sms * 8, threads = 256;
  const int iters = dtype == 0 ? 2048 : 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0);
    if (dtype == 0)
      fma_peak_kernel<double><<<blocks, threads>>>((double *)buf, iters, 0.999999, 1e-7);
    else
      fma_peak_kernel<float><<<blocks, threads>>>((float *)buf, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  if (e != cudaSuccess) return cuda_fail(e, "fma_peak_kernel");
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return KLFT_OK;
}
