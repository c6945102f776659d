// bmtab.cu -- the Box-Muller table of the FP64 exp(i eps H) proposal.
//
// The proposal's Gaussians come in pairs from the two 16-bit halves of one
// Philox word, u = (k + 1/2) 2^-16: g = r(u_a) (cos 2 pi u_b, sin 2 pi u_b) with
// r(u) = sqrt(-2 ln u).  Each half takes one of 2^16 values, so the FP64 form
// reads r and (cos, sin) from a table instead of evaluating FP64 log, sqrt and
// sincos per pair on the device.  The table is built here on the host from the
// same expressions the oracle evaluates per pair, once per device, and kept
// for the life of the process (1.5 MB).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "expprop.cuh"
#include "kernels.cuh"

namespace klft {

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_bm_mu;
const double *g_bm[kMaxDevices] = {};
}  // namespace

const double *bm_table() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_bm_mu);
  if (g_bm[dev]) return g_bm[dev];
  std::vector<double> h(3 * (size_t)BM_TAB);
  for (int k = 0; k < BM_TAB; ++k) {
    const double u = ((double)k + 0.5) * 0x1.0p-16;
    h[k] = std::sqrt(-2.0 * std::log(u));
    h[BM_TAB + 2 * k] = std::cos(6.283185307179586 * u);
    h[BM_TAB + 2 * k + 1] = std::sin(6.283185307179586 * u);
  }
  void *p = nullptr;
  if (cudaMalloc(&p, h.size() * sizeof(double)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(p);
    return nullptr;
  }
  g_bm[dev] = (const double *)p;
  return g_bm[dev];
}

}  // namespace klft
