// noalloc.cu -- Metropolis sweeps that allocate nothing.
//
// klft_metropolis_sweeps keeps its per-sweep acceptance counters in scratch that
// the handle allocates on first use (cudaMalloc).  Some callers cannot let the
// library allocate at that point: an application that has handed the device
// memory it may use to its own pool (a late cudaMalloc then fails), or a
// latency-critical loop that must not pay cudaMalloc/cudaFree, which can
// synchronise the whole device and stall the caller's other streams.  For them
// klft_metropolis_sweeps_noalloc runs the same sweep kernels with the counters
// in a fixed, file-scope device array instead.
//
// The array holds KLFT_NOALLOC_MAX_SWEEPS counters (8 KB) and lives on every GPU
// that loads the library until the process exits.  Host code never touches the
// array's name as an address: on the first call on a device (with that device
// current) the entry point asks the runtime for the array's device address with
// cudaGetSymbolAddress and keeps it for later calls on that device.  That first
// call should therefore come before any stream capture.  The first call on a
// device may also make the CUDA driver load this library's kernels (lazy module
// loading), which can allocate driver memory once; a warm-up call after the
// lattice is created leaves every later call allocation-free.
//
// All calls on a device share the array and it keeps the last call's contents:
// each call clears the counters it uses before the sweeps.  Two calls whose GPU
// work overlapped would race on the counters, so the entry point holds a
// per-device lock from the clear until its stream has finished.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/klft_b200.h"
#include "capi_internal.h"
#include "kernels.cuh"

using namespace klft;

static __device__ __align__(256) unsigned long long g_noalloc_accepts[KLFT_NOALLOC_MAX_SWEEPS];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_setup;
std::mutex g_noalloc_device_lock[kMaxDevices];
unsigned long long *g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_accepts on the current device (set up once per device).
klft_status noalloc_counters(int dev, unsigned long long **out) {
  std::lock_guard<std::mutex> g(g_noalloc_setup);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_accepts);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_accepts)");
    g_noalloc_addr[dev] = (unsigned long long *)p;
  }
  *out = g_noalloc_addr[dev];
  return KLFT_OK;
}
}  // namespace

extern "C" klft_status klft_metropolis_sweeps_noalloc(klft_lattice *lat, double beta, double delta, int nhits,
                                                      int proposal, double eps, int nsweeps, double *acc_out) {
  if (!lat) return fail(KLFT_EINVAL, "klft_metropolis_sweeps_noalloc: null handle");
  if (nhits < 0 || nsweeps < 0) return fail(KLFT_EINVAL, "klft_metropolis_sweeps_noalloc: negative count");
  if (nsweeps > KLFT_NOALLOC_MAX_SWEEPS)
    return fail(KLFT_EINVAL,
                "klft_metropolis_sweeps_noalloc: nsweeps = %d exceeds the static maximum of %d sweeps per call "
                "(split the run into several calls)",
                nsweeps, KLFT_NOALLOC_MAX_SWEEPS);
  klft_status v = check_proposal(lat, delta, proposal, eps, "klft_metropolis_sweeps_noalloc");
  if (v != KLFT_OK) return v;
  if (nsweeps == 0) return KLFT_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != lat->device)
    return fail(KLFT_EINVAL, "klft_metropolis_sweeps_noalloc: current device %d is not the lattice's device %d", dev,
                lat->device);
  if (dev < 0 || dev >= kMaxDevices) return fail(KLFT_EINVAL, "klft_metropolis_sweeps_noalloc: device %d", dev);
  unsigned long long *d_acc = nullptr;
  klft_status s = noalloc_counters(dev, &d_acc);
  if (s != KLFT_OK) return s;

  std::lock_guard<std::mutex> hold(g_noalloc_device_lock[dev]);
  std::lock_guard<std::mutex> guard(lat->mtx);
  const size_t bytes = (size_t)nsweeps * sizeof(unsigned long long);
  e = cudaMemsetAsync(d_acc, 0, bytes, lat->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(static counters)");
  // may_tune = false: a launch shape the tuner already chose is used, but no
  // tuning (which would allocate a scratch copy of the links) starts here
  s = enqueue_sweeps(lat, beta, delta, nhits, proposal, eps, nsweeps, d_acc, lat->defect, false);
  if (s != KLFT_OK) {
    cudaStreamSynchronize(lat->stream);
    return s;
  }
  if (acc_out) {
    // the counts land in the caller's buffer (8 bytes each) and are turned into
    // acceptance rates in place: no host or device allocation
    e = cudaMemcpyAsync(acc_out, d_acc, bytes, cudaMemcpyDeviceToHost, lat->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(lat->stream);
    if (e != cudaSuccess) return cuda_fail(e, "klft_metropolis_sweeps_noalloc: read back");
    double norm = 1.0;
    for (int d = 0; d < lat->g.nd; ++d) norm *= (double)lat->g.L[d];
    norm *= (double)lat->g.nd;
    norm *= (double)nhits;
    for (int k = 0; k < nsweeps; ++k) {
      unsigned long long c;
      memcpy(&c, &acc_out[k], sizeof c);
      acc_out[k] = nhits > 0 ? (double)c / norm : 0.0;
    }
  } else {
    e = cudaStreamSynchronize(lat->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
  }
  return KLFT_OK;
}
