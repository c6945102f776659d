// capi.cu -- the extern "C" boundary of libklft_b200.so (declared in
// include/klft_b200.h): lattice handles, their streams and scratch, and the
// host-side sequencing of the kernels (sweep = 2^Nd parity-class passes).
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/klft_b200.h"
#include "capi_internal.h"
#include "kernels.cuh"
#include "tuner.h"

using namespace klft;

namespace klft {

static thread_local std::string g_last_error;

klft_status fail(klft_status code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

klft_status cuda_fail(cudaError_t e, const char *what) {
  return fail(e == cudaErrorMemoryAllocation ? KLFT_ENOMEM : KLFT_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

cudaError_t Scratch::ensure(size_t bytes) {
  if (bytes <= cap) return cudaSuccess;
  release();
  cudaError_t e = stream ? cudaMallocAsync(&ptr, bytes, stream) : cudaMalloc(&ptr, bytes);
  if (e == cudaSuccess) cap = bytes;
  else ptr = nullptr;
  return e;
}
void Scratch::release() {
  if (ptr) {
    if (stream) cudaFreeAsync(ptr, stream);
    else cudaFree(ptr);
  }
  ptr = nullptr;
  cap = 0;
}

namespace {
std::mutex g_pin_mu;
std::vector<double *> g_pin_free;
std::mutex g_pool_mu;
std::vector<int> g_pool_done;
}  // namespace

double *pinned_slots_get() {
  {
    std::lock_guard<std::mutex> g(g_pin_mu);
    if (!g_pin_free.empty()) {
      double *p = g_pin_free.back();
      g_pin_free.pop_back();
      return p;
    }
  }
  double *p = nullptr;
  if (cudaMallocHost(&p, KLFT_RESULT_SLOTS * sizeof(double)) != cudaSuccess) return nullptr;
  return p;
}

void pinned_slots_put(double *p) {
  if (!p) return;
  std::lock_guard<std::mutex> g(g_pin_mu);
  g_pin_free.push_back(p);
}

void keep_pool_memory(int device) {
  std::lock_guard<std::mutex> g(g_pool_mu);
  for (int d : g_pool_done)
    if (d == device) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  g_pool_done.push_back(device);
}

}  // namespace klft

#define CK(call)                                           \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);    \
  } while (0)

#define LOCK(lat) std::lock_guard<std::mutex> guard_((lat)->mtx)

static size_t elem_bytes(int precision) { return precision == KLFT_PRECISION_FP64 ? 16 : 8; }

klft_status klft::lattice_sync(klft_lattice *lat) {
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

// Proposal arguments: the reference SU(3) generator needs delta > 0 (its
// rejection loops draw from [0, delta) until the norm is nonzero).
klft_status klft::check_proposal(const klft_lattice *lat, double delta, int proposal, double eps, const char *who) {
  if (proposal != KLFT_PROPOSAL_REFERENCE && proposal != KLFT_PROPOSAL_EXP)
    return fail(KLFT_EINVAL, "%s: unknown proposal %d", who, proposal);
  if (!(delta == delta) || !(eps == eps)) return fail(KLFT_EINVAL, "%s: NaN step size", who);
  if (lat->nc == 3 && proposal == KLFT_PROPOSAL_REFERENCE && !(delta > 0.0))
    return fail(KLFT_EINVAL, "%s: the reference SU(3) proposal needs delta > 0 (got %g)", who, delta);
  return KLFT_OK;
}

namespace klft {
// extents already checked (even, >= 2, volume < 2^31)
Geom make_geom(int ndims, const int *L) {
  Geom g{};
  g.nd = ndims;
  long long V = 1, Vh = 1;
  int stride = 1;
  for (int d = 0; d < 4; ++d) {
    g.L[d] = d < ndims ? L[d] : 1;
    g.H[d] = d < ndims ? L[d] / 2 : 1;
    g.hs[d] = stride;
    stride *= g.H[d];
    Vh *= g.H[d];
    if (d < ndims) V *= L[d];
  }
  g.V = V;
  g.Vh = Vh;
  g.open_mu = -1;
  return g;
}
}  // namespace klft

extern "C" {

const char *klft_last_error(void) { return g_last_error.c_str(); }

int klft_version(void) { return 100; }

klft_status klft_device_count(int *n) {
  if (!n) return fail(KLFT_EINVAL, "klft_device_count: null pointer");
  cudaError_t e = cudaGetDeviceCount(n);
  if (e != cudaSuccess) {
    *n = 0;
    return cuda_fail(e, "cudaGetDeviceCount");
  }
  return KLFT_OK;
}

klft_status klft_set_device(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(KLFT_ECUDA, "klft_set_device: no CUDA device available");
  if (device < 0 || device >= n) return fail(KLFT_EINVAL, "klft_set_device: no device %d (%d present)", device, n);
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  return KLFT_OK;
}

klft_status klft_lattice_create(int nc, int ndims, const int *L, int precision, int start, uint64_t seed,
                                klft_lattice **out) {
  if (!out || !L) return fail(KLFT_EINVAL, "klft_lattice_create: null pointer");
  *out = nullptr;
  if (nc < 1 || nc > 3) return fail(KLFT_EINVAL, "klft_lattice_create: Nc must be 1, 2 or 3 (got %d)", nc);
  if (ndims < 2 || ndims > 4) return fail(KLFT_EINVAL, "klft_lattice_create: ndims must be 2, 3 or 4 (got %d)", ndims);
  if (precision != KLFT_PRECISION_FP64 && precision != KLFT_PRECISION_MIXED)
    return fail(KLFT_EINVAL, "klft_lattice_create: unknown precision %d", precision);
  if (start != KLFT_START_COLD && start != KLFT_START_HOT)
    return fail(KLFT_EINVAL, "klft_lattice_create: unknown start %d", start);
  long long V = 1;
  for (int d = 0; d < ndims; ++d) {
    if (L[d] < 2 || (L[d] & 1))
      return fail(KLFT_EINVAL, "klft_lattice_create: extent L%d = %d must be even and >= 2", d, L[d]);
    V *= L[d];
  }
  if (V > 0x7fffffffLL) return fail(KLFT_EINVAL, "klft_lattice_create: volume %lld exceeds 2^31-1", V);
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(KLFT_ECUDA, "klft_lattice_create: no CUDA device available");

  klft_lattice *lat = new klft_lattice();
  lat->nc = nc;
  lat->precision = precision;
  lat->seed = seed;
  lat->chain = 0;
  lat->g = make_geom(ndims, L);
  const Geom &g = lat->g;
  cudaGetDevice(&lat->device);
  lat->link_bytes = (size_t)V * ndims * link_planes(nc, lat->dtype()) * elem_bytes(precision);
  e = cudaStreamCreateWithFlags(&lat->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete lat; return cuda_fail(e, "cudaStreamCreate"); }
  keep_pool_memory(lat->device);
  for (Scratch *sc : {&lat->s_part, &lat->s_out, &lat->s_aux, &lat->s_stage, &lat->s_wl, &lat->s_hmc, &lat->s_gf,
                      &lat->s_tab, &lat->s_tune})
    sc->stream = lat->stream;
  e = cudaMallocAsync(&lat->links, lat->link_bytes, lat->stream);
  if (e != cudaSuccess) {
    lat->links = nullptr;
    klft_status st = cuda_fail(e, "cudaMallocAsync(links)");
    klft_lattice_destroy(lat);
    return st;
  }
  e = cudaMallocAsync(&lat->d_counters, 4 * sizeof(uint32_t), lat->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(lat->d_counters, 0, 4 * sizeof(uint32_t), lat->stream);
  if (e == cudaSuccess) {
    lat->h_results = pinned_slots_get();
    if (!lat->h_results) e = cudaErrorMemoryAllocation;
  }
  if (e == cudaSuccess)
    e = launch_init(nc, precision == KLFT_PRECISION_FP64 ? 0 : 1, lat->links, g, start == KLFT_START_HOT, seed, 0,
                    lat->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lat->stream);
  // the FP64 SU(3) exp proposal's Box-Muller table, built here so that no
  // sweep (captured into a graph or not) has to allocate it
  if (e == cudaSuccess && nc == 3 && precision == KLFT_PRECISION_FP64 && !bm_table()) e = cudaErrorMemoryAllocation;
  if (e != cudaSuccess) {
    klft_status s = cuda_fail(e, "klft_lattice_create");
    klft_lattice_destroy(lat);
    return s;
  }
  *out = lat;
  return KLFT_OK;
}

klft_status klft_lattice_destroy(klft_lattice *lat) {
  if (!lat) return KLFT_OK;
  {
    LOCK(lat);
    if (lat->stream) cudaStreamSynchronize(lat->stream);
    for (Scratch *s : {&lat->s_part, &lat->s_out, &lat->s_aux, &lat->s_stage, &lat->s_wl, &lat->s_hmc,
                        &lat->s_gf, &lat->s_tab, &lat->s_tune})
      s->release();
    // stream-ordered frees: no device-wide synchronisation
    if (lat->links) cudaFreeAsync(lat->links, lat->stream);
    if (lat->d_counters) cudaFreeAsync(lat->d_counters, lat->stream);
    pinned_slots_put(lat->h_results);
    if (lat->side) {
      cudaStreamSynchronize(lat->side);
      cudaStreamDestroy(lat->side);
    }
    for (cudaEvent_t ev : {lat->ev_fork, lat->ev_join, lat->ev_up, lat->ev_loops})
      if (ev) cudaEventDestroy(ev);
    if (lat->stream) cudaStreamDestroy(lat->stream);
  }
  delete lat;
  return KLFT_OK;
}

klft_status klft_lattice_info(const klft_lattice *lat, int *nc, int *ndims, int *L, int *precision,
                              long long *volume) {
  if (!lat) return fail(KLFT_EINVAL, "klft_lattice_info: null handle");
  if (nc) *nc = lat->nc;
  if (ndims) *ndims = lat->g.nd;
  if (L)
    for (int d = 0; d < lat->g.nd; ++d) L[d] = lat->g.L[d];
  if (precision) *precision = lat->precision;
  if (volume) *volume = lat->g.V;
  return KLFT_OK;
}

klft_status klft_lattice_set_stream(klft_lattice *lat, uint64_t seed, uint64_t chain) {
  if (!lat) return fail(KLFT_EINVAL, "klft_lattice_set_stream: null handle");
  LOCK(lat);
  lat->seed = seed;
  lat->chain = chain;
  return KLFT_OK;
}

klft_status klft_lattice_get_counters(klft_lattice *lat, uint32_t *sweep, uint32_t *trajectory) {
  if (!lat) return fail(KLFT_EINVAL, "klft_lattice_get_counters: null handle");
  LOCK(lat);
  uint32_t c[4];
  CK(cudaMemcpyAsync(c, lat->d_counters, sizeof c, cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  if (sweep) *sweep = c[0];
  if (trajectory) *trajectory = c[1];
  return KLFT_OK;
}

klft_status klft_lattice_set_counters(klft_lattice *lat, uint32_t sweep, uint32_t trajectory) {
  if (!lat) return fail(KLFT_EINVAL, "klft_lattice_set_counters: null handle");
  LOCK(lat);
  uint32_t c[4] = {sweep, trajectory, 0, 0};
  CK(cudaMemcpyAsync(lat->d_counters, c, sizeof c, cudaMemcpyHostToDevice, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_lattice_upload(klft_lattice *lat, const double *host) {
  if (!lat || !host) return fail(KLFT_EINVAL, "klft_lattice_upload: null pointer");
  LOCK(lat);
  const size_t nlinks = (size_t)lat->g.V * lat->g.nd;
  if (lat->dtype() == 1) {
    // mixed form: the host rounds the stored reals to FP32, a third of the bytes cross PCIe for SU(3)
    CK(lat->s_stage.ensure(nlinks * link_planes(lat->nc, 1) * 2 * sizeof(float)));
    CK(upload_links_f32(lat->s_stage.ptr, host, nlinks, lat->nc, lat->stream));
    CK(launch_import_f32(lat->nc, lat->links, lat->g, (const float *)lat->s_stage.ptr, lat->stream));
  } else {
    const size_t bytes = nlinks * lat->nc * lat->nc * 16;
    CK(lat->s_stage.ensure(bytes));
    CK(copy_host_to_device(lat->s_stage.ptr, host, bytes, lat->stream));
    CK(launch_import(lat->nc, lat->dtype(), lat->links, lat->g, (const double *)lat->s_stage.ptr, lat->stream));
  }
  CK(launch_open_boundary(lat->nc, lat->dtype(), lat->links, lat->g, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_lattice_set_open_boundary(klft_lattice *lat, int mu) {
  if (!lat) return fail(KLFT_EINVAL, "klft_lattice_set_open_boundary: null handle");
  if (mu < -1 || mu >= lat->g.nd)
    return fail(KLFT_EINVAL, "klft_lattice_set_open_boundary: direction %d outside -1..%d", mu, lat->g.nd - 1);
  LOCK(lat);
  if (mu < 0 && lat->g.open_mu >= 0)
    return fail(KLFT_EINVAL, "klft_lattice_set_open_boundary: the zeroed boundary links cannot be restored; "
                             "upload a configuration into a new lattice instead");
  if (mu >= 0 && lat->g.open_mu >= 0 && mu != lat->g.open_mu)
    return fail(KLFT_EINVAL, "klft_lattice_set_open_boundary: direction %d is already open", lat->g.open_mu);
  lat->g.open_mu = mu;
  CK(launch_open_boundary(lat->nc, lat->dtype(), lat->links, lat->g, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_lattice_download(klft_lattice *lat, double *host) {
  if (!lat || !host) return fail(KLFT_EINVAL, "klft_lattice_download: null pointer");
  LOCK(lat);
  const size_t nlinks = (size_t)lat->g.V * lat->g.nd;
  if (lat->dtype() == 1) {
    // mixed form: the stored FP32 reals cross PCIe, the host completes each link in FP64
    CK(lat->s_stage.ensure(nlinks * link_planes(lat->nc, 1) * 2 * sizeof(float)));
    CK(launch_export_f32(lat->nc, lat->links, lat->g, (float *)lat->s_stage.ptr, lat->stream));
    CK(download_links_f32(host, lat->s_stage.ptr, nlinks, lat->nc, lat->stream));
  } else {
    const size_t bytes = nlinks * lat->nc * lat->nc * 16;
    CK(lat->s_stage.ensure(bytes));
    CK(launch_export(lat->nc, lat->dtype(), lat->links, lat->g, (double *)lat->s_stage.ptr, lat->stream));
    CK(copy_device_to_host(host, lat->s_stage.ptr, bytes, lat->stream));
  }
  return KLFT_OK;
}

klft_status klft_metropolis_sweeps(klft_lattice *lat, double beta, double delta, int nhits, int proposal, double eps,
                                   int nsweeps, double *acc_out) {
  if (!lat) return fail(KLFT_EINVAL, "klft_metropolis_sweeps: null handle");
  if (nhits < 0 || nsweeps < 0) return fail(KLFT_EINVAL, "klft_metropolis_sweeps: negative count");
  klft_status v = check_proposal(lat, delta, proposal, eps, "klft_metropolis_sweeps");
  if (v != KLFT_OK) return v;
  if (nsweeps == 0) return KLFT_OK;
  LOCK(lat);
  CK(lat->s_aux.ensure((size_t)nsweeps * sizeof(unsigned long long)));
  unsigned long long *d_nacc = (unsigned long long *)lat->s_aux.ptr;
  CK(cudaMemsetAsync(d_nacc, 0, (size_t)nsweeps * sizeof(unsigned long long), lat->stream));
  klft_status s = enqueue_sweeps(lat, beta, delta, nhits, proposal, eps, nsweeps, d_nacc, lat->defect);
  if (s != KLFT_OK) return s;
  if (acc_out) {
    std::vector<unsigned long long> h(nsweeps);
    CK(cudaMemcpyAsync(h.data(), d_nacc, (size_t)nsweeps * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       lat->stream));
    CK(cudaStreamSynchronize(lat->stream));
    double norm = 1.0;
    for (int d = 0; d < lat->g.nd; ++d) norm *= (double)lat->g.L[d];
    norm *= (double)lat->g.nd;
    norm *= (double)nhits;
    for (int k = 0; k < nsweeps; ++k) acc_out[k] = nhits > 0 ? (double)h[k] / norm : 0.0;
  } else {
    CK(cudaStreamSynchronize(lat->stream));
  }
  return KLFT_OK;
}

klft_status klft_plaquette(klft_lattice *lat, double *out) {
  if (!lat || !out) return fail(KLFT_EINVAL, "klft_plaquette: null pointer");
  LOCK(lat);
  klft_status s = enqueue_plaquette(lat, 0);
  if (s != KLFT_OK) return s;
  CK(cudaMemcpyAsync(lat->h_results, lat->s_out.ptr, sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  *out = normalize_plaquette(lat, lat->h_results[0]);
  return KLFT_OK;
}

klft_status klft_wilson_loop_mu_nu(klft_lattice *lat, int mu, int nu, const int *pairs, int npairs, double *out) {
  if (!lat || (npairs > 0 && (!pairs || !out))) return fail(KLFT_EINVAL, "klft_wilson_loop_mu_nu: null pointer");
  if (mu < 0 || nu < 0 || mu >= lat->g.nd || nu >= lat->g.nd || mu == nu)
    return fail(KLFT_EINVAL, "klft_wilson_loop_mu_nu: bad plane (%d, %d)", mu, nu);
  for (int k = 0; k < npairs; ++k)
    if (pairs[2 * k] < 0 || pairs[2 * k + 1] < 0)
      return fail(KLFT_EINVAL, "klft_wilson_loop_mu_nu: negative loop extent");
  if (npairs == 0) return KLFT_OK;
  LOCK(lat);
  std::vector<double> sums(npairs);
  klft_status s = wilson_sums(lat, mu, nu, pairs, npairs, sums.data());
  if (s != KLFT_OK) return s;
  for (int k = 0; k < npairs; ++k) out[k] = normalize_wilson(lat, sums[k]);
  return KLFT_OK;
}

klft_status klft_wilson_loop_temporal(klft_lattice *lat, const int *pairs, int npairs, double *out) {
  if (!lat || (npairs > 0 && (!pairs || !out))) return fail(KLFT_EINVAL, "klft_wilson_loop_temporal: null pointer");
  for (int k = 0; k < npairs; ++k)
    if (pairs[2 * k] < 0 || pairs[2 * k + 1] < 0)
      return fail(KLFT_EINVAL, "klft_wilson_loop_temporal: negative loop extent");
  if (npairs == 0) return KLFT_OK;
  LOCK(lat);
  const int nd = lat->g.nd;
  // one plan and one axial-gauge transformation along nu = Nd-1 for all spatial
  // planes; a single copy of the (Nd-1) x npairs sums at the end
  const size_t nsum = (size_t)(nd - 1) * npairs;
  CK(lat->s_out.ensure((nsum > KLFT_RESULT_SLOTS ? nsum : KLFT_RESULT_SLOTS) * sizeof(double)));
  WilsonPlan plan;
  klft_status s = make_wilson_plan(lat, pairs, npairs, nd - 1, plan, 0, nd - 1);
  if (s != KLFT_OK) return s;
  s = enqueue_wilson_spatial(lat, plan, false, (double *)lat->s_out.ptr, npairs);
  if (s != KLFT_OK) return s;
  std::vector<double> sums(nsum);
  CK(cudaMemcpyAsync(sums.data(), lat->s_out.ptr, nsum * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  for (int k = 0; k < npairs; ++k) {
    double acc = 0.0;
    for (int mu = 0; mu < nd - 1; ++mu) {
      const double w = normalize_wilson(lat, sums[(size_t)mu * npairs + k]);
      acc = mu == 0 ? w : acc + w;
    }
    out[k] = acc / (double)(nd - 1);
  }
  return KLFT_OK;
}

klft_status klft_staple_field(klft_lattice *lat, double *out) {
  if (!lat || !out) return fail(KLFT_EINVAL, "klft_staple_field: null pointer");
  LOCK(lat);
  const size_t bytes = (size_t)lat->g.V * lat->g.nd * lat->nc * lat->nc * 16;
  CK(lat->s_stage.ensure(bytes));
  CK(launch_staple_field(lat->nc, lat->dtype(), lat->links, lat->g, (double *)lat->s_stage.ptr, lat->stream));
  CK(cudaMemcpyAsync(out, lat->s_stage.ptr, bytes, cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_unitarity(klft_lattice *lat, double *out) {
  if (!lat || !out) return fail(KLFT_EINVAL, "klft_unitarity: null pointer");
  LOCK(lat);
  CK(lat->s_part.ensure(4096 * sizeof(double)));
  CK(lat->s_out.ensure(KLFT_RESULT_SLOTS * sizeof(double)));
  CK(launch_unitarity(lat->nc, lat->dtype(), lat->links, lat->g, (double *)lat->s_part.ptr, (double *)lat->s_out.ptr,
                      lat->stream));
  CK(cudaMemcpyAsync(lat->h_results, lat->s_out.ptr, sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  *out = lat->h_results[0];
  return KLFT_OK;
}

klft_status klft_reunitarize(klft_lattice *lat) {
  if (!lat) return fail(KLFT_EINVAL, "klft_reunitarize: null handle");
  LOCK(lat);
  CK(launch_reunitarize(lat->nc, lat->dtype(), lat->links, lat->g, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_run_cycles(klft_lattice *lat, double beta, double delta, int nhits, int proposal, double eps,
                            int ncycles, int measure_plaquette, const int *temporal_pairs, int npairs,
                            double *acc_out, double *plaq_out, double *w_out, double *device_ms) {
  if (!lat) return fail(KLFT_EINVAL, "klft_run_cycles: null handle");
  if (ncycles < 0 || nhits < 0 || npairs < 0) return fail(KLFT_EINVAL, "klft_run_cycles: negative count");
  if (npairs > 0 && !temporal_pairs) return fail(KLFT_EINVAL, "klft_run_cycles: null pairs");
  klft_status v = check_proposal(lat, delta, proposal, eps, "klft_run_cycles");
  if (v != KLFT_OK) return v;
  for (int k = 0; k < npairs; ++k)
    if (temporal_pairs[2 * k] < 0 || temporal_pairs[2 * k + 1] < 0)
      return fail(KLFT_EINVAL, "klft_run_cycles: negative loop extent");
  if (ncycles == 0) return KLFT_OK;
  LOCK(lat);
  const int nd = lat->g.nd;
  const int nw = (nd - 1) * npairs;  // per cycle: one sum per (spatial mu, pair)
  // wl: [nacc ncycles (u64)][plaq ncycles][w ncycles*nw], one block so that one
  // copy brings the results back, then the plaquette's block partials (the loop
  // kernels, which may run at the same time, keep theirs in s_part); all
  // scratch sized before the first launch
  const size_t nres = (size_t)ncycles * (2 + nw);  // 8-byte slots
  const int nblk_plaq = plaquette_blocks(lat->g);
  CK(lat->s_wl.ensure((nres + (size_t)nblk_plaq) * sizeof(double)));
  unsigned long long *d_nacc = (unsigned long long *)lat->s_wl.ptr;
  double *d_plaq = (double *)lat->s_wl.ptr + ncycles;
  double *d_w = d_plaq + ncycles;
  double *d_plaq_part = (double *)lat->s_wl.ptr + nres;
  WilsonPlan plan;
  if (npairs > 0) {
    klft_status s = make_wilson_plan(lat, temporal_pairs, npairs, nd - 1, plan, 0, nd - 1);
    if (s != KLFT_OK) return s;
  }
  // With loops to measure, two parts of a cycle run on the side stream: the
  // plaquette (it reads every link) beside the loops' axial-gauge
  // transformation (one thread per column: a latency-bound kernel that leaves
  // most of the device idle), and the gauge-fixed form's loop kernels, which
  // read only U', beside the next cycle's sweep.  Events order the rest: the
  // next sweep waits for the plaquette, the next U' for the loops.
  const bool fork = measure_plaquette && npairs > 0;
  const bool loops_side = npairs > 0 && plan.gf;
  if ((fork || loops_side) && !lat->side) {
    CK(cudaStreamCreateWithFlags(&lat->side, cudaStreamNonBlocking));
    for (cudaEvent_t *ev : {&lat->ev_fork, &lat->ev_join, &lat->ev_up, &lat->ev_loops})
      CK(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  }
  // on an early return: the main stream after everything enqueued on the side stream
  auto join_side = [&] {
    if ((fork || loops_side) && cudaEventRecord(lat->ev_join, lat->side) == cudaSuccess)
      cudaStreamWaitEvent(lat->stream, lat->ev_join, 0);
  };
  CK(cudaMemsetAsync(d_nacc, 0, (size_t)ncycles * sizeof(unsigned long long), lat->stream));
  // The temporal (1, 1) loop of plane (mu, Nd-1) is that plane's plaquette: when
  // the pair list holds it, the plaquette kernel covers the spatial planes only
  // and the temporal planes come from the loop sums (added in FP64 below).
  int k11 = -1;
  for (int k = 0; k < npairs && k11 < 0; ++k)
    if (temporal_pairs[2 * k] == 1 && temporal_pairs[2 * k + 1] == 1) k11 = k;
  const int plaq_nu_end = k11 >= 0 ? nd - 1 : nd;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, lat->stream));
  for (int c = 0; c < ncycles; ++c) {
    klft_status s = enqueue_sweeps(lat, beta, delta, nhits, proposal, eps, 1, d_nacc + c, lat->defect);
    cudaError_t e = cudaSuccess;
    if (s == KLFT_OK && fork) {
      e = cudaEventRecord(lat->ev_fork, lat->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(lat->side, lat->ev_fork, 0);
    }
    if (s == KLFT_OK && e == cudaSuccess && measure_plaquette)
      e = launch_plaquette(lat->nc, lat->dtype(), lat->links, lat->g, d_plaq_part, nblk_plaq, d_plaq + c,
                           fork ? lat->side : lat->stream, plaq_nu_end);
    if (s == KLFT_OK && e == cudaSuccess && fork) e = cudaEventRecord(lat->ev_join, lat->side);
    // U' of this cycle after the loops of the previous one
    if (s == KLFT_OK && e == cudaSuccess && loops_side && c > 0)
      e = cudaStreamWaitEvent(lat->stream, lat->ev_loops, 0);
    if (s == KLFT_OK && e == cudaSuccess && npairs > 0) {
      // the spatial planes share the axial-gauge transformation along nu = Nd-1
      s = enqueue_wilson_spatial(lat, plan, false, d_w + (size_t)c * nw, npairs, loops_side ? lat->side : nullptr,
                                 lat->ev_up);
      if (s == KLFT_OK && loops_side) e = cudaEventRecord(lat->ev_loops, lat->side);
    }
    // the next sweep after the plaquette
    if (s == KLFT_OK && e == cudaSuccess && fork) e = cudaStreamWaitEvent(lat->stream, lat->ev_join, 0);
    if (s != KLFT_OK || e != cudaSuccess) {
      join_side();
      return s != KLFT_OK ? s : cuda_fail(e, "klft_run_cycles");
    }
  }
  // the result copy after the last loops
  if (loops_side) CK(cudaStreamWaitEvent(lat->stream, lat->ev_loops, 0));
  CK(cudaEventRecord(e1, lat->stream));
  // into the handle's page-locked slots when the results fit (one DMA copy)
  std::vector<double> h_big;
  double *h_res = lat->h_results;
  if (nres > KLFT_RESULT_SLOTS) {
    h_big.resize(nres);
    h_res = h_big.data();
  }
  CK(cudaMemcpyAsync(h_res, lat->s_wl.ptr, nres * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  const unsigned long long *h_nacc = (const unsigned long long *)h_res;
  const double *h_out = h_res + ncycles;
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (device_ms) *device_ms = ms;
  double norm = 1.0;
  for (int d = 0; d < nd; ++d) norm *= (double)lat->g.L[d];
  norm *= (double)nd;
  norm *= (double)nhits;
  for (int c = 0; c < ncycles; ++c) {
    if (acc_out) acc_out[c] = nhits > 0 ? (double)h_nacc[c] / norm : 0.0;
    if (plaq_out && measure_plaquette) {
      double sum = h_out[c];
      if (k11 >= 0)
        for (int mu = 0; mu < nd - 1; ++mu) sum += h_out[ncycles + (size_t)c * nw + (size_t)mu * npairs + k11];
      plaq_out[c] = normalize_plaquette(lat, sum);
    }
    if (w_out)
      for (int k = 0; k < npairs; ++k) {
        double acc = 0.0;
        for (int mu = 0; mu < nd - 1; ++mu) {
          const double w = normalize_wilson(lat, h_out[ncycles + (size_t)c * nw + (size_t)mu * npairs + k]);
          acc = mu == 0 ? w : acc + w;
        }
        w_out[(size_t)c * npairs + k] = acc / (double)(nd - 1);
      }
  }
  return KLFT_OK;
}

klft_status klft_run_metropolis(klft_lattice *lat, double beta, double delta, int nhits, int proposal, double eps,
                                int nsweeps, int interval, int measure_plaquette, const int *temporal_pairs,
                                int ntemporal, const int *planes, int nplanes, const int *planar_pairs, int nplanar,
                                double *acc_out, double *plaq_out, double *wtemp_out, double *wmunu_out,
                                double *device_ms) {
  const char *who = "klft_run_metropolis";
  if (!lat) return fail(KLFT_EINVAL, "%s: null handle", who);
  if (nsweeps < 0 || nhits < 0 || interval < 0 || ntemporal < 0 || nplanes < 0 || nplanar < 0)
    return fail(KLFT_EINVAL, "%s: negative count", who);
  if ((ntemporal > 0 && !temporal_pairs) || (nplanes > 0 && !planes) || (nplanar > 0 && !planar_pairs))
    return fail(KLFT_EINVAL, "%s: null list", who);
  klft_status v = check_proposal(lat, delta, proposal, eps, who);
  if (v != KLFT_OK) return v;
  const int nd = lat->g.nd;
  for (int k = 0; k < ntemporal; ++k)
    if (temporal_pairs[2 * k] < 0 || temporal_pairs[2 * k + 1] < 0)
      return fail(KLFT_EINVAL, "%s: negative loop extent", who);
  for (int k = 0; k < nplanar; ++k)
    if (planar_pairs[2 * k] < 0 || planar_pairs[2 * k + 1] < 0) return fail(KLFT_EINVAL, "%s: negative loop extent", who);
  for (int q = 0; q < nplanes; ++q) {
    const int mu = planes[2 * q], nu = planes[2 * q + 1];
    if (mu < 0 || nu < 0 || mu >= nd || nu >= nd || mu == nu) return fail(KLFT_EINVAL, "%s: bad plane (%d, %d)", who, mu, nu);
  }
  if (nsweeps == 0) return KLFT_OK;
  LOCK(lat);
  // measurements after sweeps step = interval, 2 interval, ... < nsweeps (GaugeObservable.hpp:69-73)
  const int nmeas = interval > 0 ? (nsweeps - 1) / interval : 0;
  const bool do_plaq = measure_plaquette && nmeas > 0;
  const int ntw = ntemporal > 0 && nmeas > 0 ? (nd - 1) * ntemporal : 0;  // sums per measurement
  const int npw = nplanar > 0 && nmeas > 0 ? nplanes * nplanar : 0;
  const size_t per = 1 + (size_t)ntw + (size_t)npw;
  CK(lat->s_aux.ensure((size_t)nsweeps * sizeof(unsigned long long)));
  // wl: the measurements' results, then the plaquette's block partials (apart
  // from the loop kernels', which may run at the same time)
  const int nblk_plaq = plaquette_blocks(lat->g);
  CK(lat->s_wl.ensure(((size_t)nmeas * per + 1 + (size_t)nblk_plaq) * sizeof(double)));
  unsigned long long *d_nacc = (unsigned long long *)lat->s_aux.ptr;
  double *d_res = (double *)lat->s_wl.ptr;
  double *d_plaq_part = d_res + (size_t)nmeas * per + 1;
  // plans: temporal loops along nu = Nd-1, one plan per distinct nu of the planar list
  CK(lat->s_tab.ensure((2 * (size_t)ntemporal + (size_t)nplanes * 2 * nplanar) * sizeof(int) + 16));
  WilsonPlan tplan;
  size_t toff = 0;
  if (ntw > 0) {
    klft_status s = make_wilson_plan(lat, temporal_pairs, ntemporal, nd - 1, tplan, toff);
    if (s != KLFT_OK) return s;
    toff += 2 * (size_t)ntemporal;
  }
  std::vector<WilsonPlan> pplan(npw > 0 ? nplanes : 0);
  for (int q = 0; q < (int)pplan.size(); ++q) {
    klft_status s = make_wilson_plan(lat, planar_pairs, nplanar, planes[2 * q + 1], pplan[q], toff);
    if (s != KLFT_OK) return s;
    toff += 2 * (size_t)nplanar;
  }
  // As in klft_run_cycles: the plaquette on the handle's second stream beside
  // the loops' axial-gauge transformation, and (with no planar loops, which
  // would share the loop scratch) the temporal loop kernel beside the sweeps
  // that follow; events order the rest.
  const bool fork = do_plaq && (ntw > 0 || npw > 0);
  const bool loops_side = ntw > 0 && tplan.gf && npw == 0;
  if ((fork || loops_side) && !lat->side) {
    CK(cudaStreamCreateWithFlags(&lat->side, cudaStreamNonBlocking));
    for (cudaEvent_t *ev : {&lat->ev_fork, &lat->ev_join, &lat->ev_up, &lat->ev_loops})
      CK(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  }
  auto join_side = [&] {
    if ((fork || loops_side) && cudaEventRecord(lat->ev_join, lat->side) == cudaSuccess)
      cudaStreamWaitEvent(lat->stream, lat->ev_join, 0);
  };
  CK(cudaMemsetAsync(d_nacc, 0, (size_t)nsweeps * sizeof(unsigned long long), lat->stream));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, lat->stream));
  int m = 0;
  for (int step = 0; step < nsweeps; ++step) {
    klft_status s = enqueue_sweeps(lat, beta, delta, nhits, proposal, eps, 1, d_nacc + step, lat->defect);
    if (s != KLFT_OK) {
      join_side();
      return s;
    }
    if (!(interval > 0 && step % interval == 0 && step != 0)) continue;
    double *slot = d_res + (size_t)m * per;
    cudaError_t e = cudaSuccess;
    if (fork) {
      e = cudaEventRecord(lat->ev_fork, lat->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(lat->side, lat->ev_fork, 0);
    }
    if (e == cudaSuccess && do_plaq)
      e = launch_plaquette(lat->nc, lat->dtype(), lat->links, lat->g, d_plaq_part, nblk_plaq, slot,
                           fork ? lat->side : lat->stream);
    if (e == cudaSuccess && fork) e = cudaEventRecord(lat->ev_join, lat->side);
    int last_nu = -1;
    if (e == cudaSuccess && ntw > 0) {
      // U' of this measurement after the loops of the previous one
      if (loops_side && m > 0) e = cudaStreamWaitEvent(lat->stream, lat->ev_loops, 0);
      if (e == cudaSuccess)
        s = enqueue_wilson_spatial(lat, tplan, false, slot + 1, ntemporal, loops_side ? lat->side : nullptr,
                                   lat->ev_up);
      if (e == cudaSuccess && s == KLFT_OK && loops_side) e = cudaEventRecord(lat->ev_loops, lat->side);
      last_nu = nd - 1;
    }
    for (int q = 0; q < (int)pplan.size() && s == KLFT_OK && e == cudaSuccess; ++q) {
      const int mu = planes[2 * q], nu = planes[2 * q + 1];
      s = enqueue_wilson_plane(lat, pplan[q], mu, nu, last_nu == nu, slot + 1 + ntw + (size_t)q * nplanar);
      last_nu = nu;
    }
    // the next sweep after the plaquette
    if (s == KLFT_OK && e == cudaSuccess && fork) e = cudaStreamWaitEvent(lat->stream, lat->ev_join, 0);
    if (s != KLFT_OK || e != cudaSuccess) {
      join_side();
      return s != KLFT_OK ? s : cuda_fail(e, "klft_run_metropolis");
    }
    ++m;
  }
  // the result copy after the last loops
  if (loops_side) CK(cudaStreamWaitEvent(lat->stream, lat->ev_loops, 0));
  CK(cudaEventRecord(e1, lat->stream));
  std::vector<unsigned long long> h_nacc(nsweeps);
  std::vector<double> h_res((size_t)nmeas * per);
  CK(cudaMemcpyAsync(h_nacc.data(), d_nacc, (size_t)nsweeps * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     lat->stream));
  if (!h_res.empty())
    CK(cudaMemcpyAsync(h_res.data(), d_res, h_res.size() * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (device_ms) *device_ms = ms;
  double norm = 1.0;
  for (int d = 0; d < nd; ++d) norm *= (double)lat->g.L[d];
  norm *= (double)nd * (double)nhits;
  for (int k = 0; k < nsweeps; ++k)
    if (acc_out) acc_out[k] = nhits > 0 ? (double)h_nacc[k] / norm : 0.0;
  for (int i = 0; i < nmeas; ++i) {
    const double *r = h_res.data() + (size_t)i * per;
    if (plaq_out && do_plaq) plaq_out[i] = normalize_plaquette(lat, r[0]);
    if (wtemp_out)
      for (int k = 0; k < ntemporal && ntw > 0; ++k) {
        // WilsonLoop.hpp:250-304: the average over the spatial directions mu
        double acc = 0.0;
        for (int mu = 0; mu < nd - 1; ++mu) {
          const double w = normalize_wilson(lat, r[1 + (size_t)mu * ntemporal + k]);
          acc = mu == 0 ? w : acc + w;
        }
        wtemp_out[(size_t)i * ntemporal + k] = acc / (double)(nd - 1);
      }
    if (wmunu_out)
      for (int j = 0; j < npw; ++j) wmunu_out[(size_t)i * npw + j] = normalize_wilson(lat, r[1 + ntw + j]);
  }
  return KLFT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ enqueue helpers
namespace klft {

// Block size of the sweep passes: 128 unless the tuner (KLFT_TUNING) picked
// another; candidates are timed on a scratch copy of the links.
static int sweep_block(klft_lattice *lat, const MetroArgs &a, const Defect &df, bool may_tune) {
  if (!tuner_enabled()) return 128;
  const std::string id = std::string("sweep_Metropolis_GaugeField_nc") + std::to_string(lat->nc) +
                         (lat->dtype() == 0 ? "_fp64" : "_mixed") +
                         (a.proposal == KLFT_PROPOSAL_EXP && lat->nc == 3 ? "_exp" : "_ref");
  const std::string key = tune_key(id, lat->g.nd, lat->g.H);
  auto time_fn = [&](int block) -> float {
    const size_t off = (lat->link_bytes + 255) & ~(size_t)255;
    if (lat->s_tune.ensure(off + 256) != cudaSuccess) return -1.f;
    void *copy = lat->s_tune.ptr;
    unsigned long long *dummy = (unsigned long long *)((char *)copy + off);
    if (cudaMemcpyAsync(copy, lat->links, lat->link_bytes, cudaMemcpyDeviceToDevice, lat->stream) != cudaSuccess)
      return -1.f;
    return time_launches(lat->stream, 3, [&] {
      return launch_metropolis_pass(lat->nc, lat->dtype(), copy, lat->g, 0, a, lat->d_counters, dummy, df, block,
                                    lat->stream);
    });
  };
  const int b = tuned_param(key, lat->g.nd, {32, 64, 128}, 128, time_fn, may_tune);
  lat->s_tune.release();
  return b;
}

klft_status enqueue_sweeps(klft_lattice *lat, double beta, double delta, int nhits, int proposal, double eps,
                           int nsweeps, unsigned long long *d_nacc, const Defect &df, bool may_tune) {
  MetroArgs a{beta, delta, eps, nhits, proposal, lat->seed, lat->chain};
  const int npass = metropolis_passes(lat->nc, proposal, lat->g.nd);
  const int block = sweep_block(lat, a, df, may_tune);
  for (int k = 0; k < nsweeps; ++k) {
    for (int val = 0; val < npass; ++val)
      CK(launch_metropolis_pass(lat->nc, lat->dtype(), lat->links, lat->g, val, a, lat->d_counters, d_nacc + k, df,
                                block, lat->stream));
    CK(launch_advance(lat->d_counters, lat->stream));
  }
  return KLFT_OK;
}

klft_status enqueue_plaquette(klft_lattice *lat, int slot) {
  const int nblk = plaquette_blocks(lat->g);
  CK(lat->s_part.ensure((size_t)nblk * sizeof(double)));
  CK(lat->s_out.ensure(KLFT_RESULT_SLOTS * sizeof(double)));
  CK(launch_plaquette(lat->nc, lat->dtype(), lat->links, lat->g, (double *)lat->s_part.ptr, nblk,
                      (double *)lat->s_out.ptr + slot, lat->stream));
  return KLFT_OK;
}

double normalize_plaquette(const klft_lattice *lat, double sum) {
  // GaugePlaquette.hpp:125-132
  double norm = 1.0;
  for (int d = 0; d < lat->g.nd; ++d) norm *= (double)lat->g.L[d];
  norm *= (double)((lat->g.nd * (lat->g.nd - 1) / 2) * lat->nc);
  return sum / norm;
}

double normalize_wilson(const klft_lattice *lat, double sum) {
  // WilsonLoop.hpp:233-240
  double w = sum;
  for (int d = 0; d < lat->g.nd; ++d) w /= (double)lat->g.L[d];
  w /= (double)lat->nc;
  return w;
}

// Build the device tables for a pair list: the pairs themselves (direct form)
// and, for the gauge-fixed form, the (T, pair) lists per loop length L.  All
// scratch the plane kernels need is sized here, before anything is enqueued.
klft_status make_wilson_plan(klft_lattice *lat, const int *pairs, int npairs, int nu, WilsonPlan &plan,
                             size_t tab_off, int nplanes) {
  plan = WilsonPlan();
  plan.npairs = npairs;
  plan.tab_off = tab_off;
  bool degenerate = false;
  for (int k = 0; k < npairs; ++k) {
    plan.lmax = pairs[2 * k] > plan.lmax ? pairs[2 * k] : plan.lmax;
    plan.tmax = pairs[2 * k + 1] > plan.tmax ? pairs[2 * k + 1] : plan.tmax;
    if (pairs[2 * k] == 0 || pairs[2 * k + 1] == 0) degenerate = true;
  }
  const size_t smem = wilson_gf_smem(lat->nc, lat->dtype(), lat->g, nu, plan.tmax, npairs);
  plan.gf = !degenerate && npairs > 0 && npairs <= WL_MAXP && plan.lmax <= WL_MAXP && plan.tmax <= 32767 &&
            smem <= 200 * 1024;
  std::vector<int> h(pairs, pairs + 2 * npairs);
  if (plan.gf) {
    plan.off.assign(plan.lmax + 2, 0);
    for (int L = 1; L <= plan.lmax; ++L) {
      plan.off[L] = (int)plan.T.size();
      for (int k = 0; k < npairs; ++k)
        if (pairs[2 * k] == L) {
          plan.T.push_back(pairs[2 * k + 1]);
          plan.p.push_back(k);
        }
    }
    plan.off[plan.lmax + 1] = (int)plan.T.size();
    CK(lat->s_gf.ensure(wilson_gf_scratch(lat->nc, lat->dtype(), lat->g, nu, plan.tmax, nplanes)));
  }
  if (!plan.gf) {
    // only the direct form reads the pairs on the device (the gauge-fixed form
    // takes its tables in the kernel parameters): no copy, and no wait, otherwise
    CK(lat->s_tab.ensure((tab_off + h.size()) * sizeof(int) + 16));
    CK(cudaMemcpyAsync((int *)lat->s_tab.ptr + tab_off, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice,
                       lat->stream));
    CK(cudaStreamSynchronize(lat->stream));  // h is pageable and local
  }
  const int nblk = plan.gf ? wilson_gf_blocks(lat->g) : plaquette_blocks(lat->g);
  CK(lat->s_part.ensure((size_t)nblk * (npairs > 1 ? npairs : 1) * (size_t)nplanes * sizeof(double)));
  return KLFT_OK;
}

// enqueue: d_out[k] = unnormalised sum over sites of Re Tr W for pair k of the plan
klft_status enqueue_wilson_plane(klft_lattice *lat, const WilsonPlan &plan, int mu, int nu, bool omega_ready,
                                 double *d_out) {
  if (plan.gf) {
    const int *ht[3] = {plan.off.data(), plan.T.data(), plan.p.data()};
    CK(launch_wilson_gf(lat->nc, lat->dtype(), lat->links, lat->g, &mu, 1, nu, ht, plan.lmax, plan.tmax,
                        plan.npairs, omega_ready, lat->s_gf.ptr, (double *)lat->s_part.ptr, wilson_gf_blocks(lat->g),
                        d_out, plan.npairs, lat->stream));
  } else {
    const int *tab = (const int *)lat->s_tab.ptr + plan.tab_off;
    const int nblk = plaquette_blocks(lat->g);
    CK(launch_wilson_direct(lat->nc, lat->dtype(), lat->links, lat->g, mu, nu, tab, plan.npairs,
                            (double *)lat->s_part.ptr, nblk, d_out, lat->stream));
  }
  return KLFT_OK;
}

// enqueue the planes (mu, Nd-1), mu < Nd-1, of a plan made with nplanes = Nd-1:
// d_out[mu * out_stride + k] = unnormalised sum for pair k; the gauge-fixed form
// runs all planes in one loop-kernel launch (one tile queue, so the last wave of
// one plane does not idle while the next plane waits for its own launch).
klft_status enqueue_wilson_spatial(klft_lattice *lat, const WilsonPlan &plan, bool omega_ready, double *d_out,
                                   int out_stride, cudaStream_t side, cudaEvent_t ev) {
  const int nu = lat->g.nd - 1;
  if (plan.gf) {
    const int *ht[3] = {plan.off.data(), plan.T.data(), plan.p.data()};
    int mus[3] = {0, 1, 2};
    // planes mu = 0 .. nu - 1
    CK(launch_wilson_gf(lat->nc, lat->dtype(), lat->links, lat->g, mus, nu, nu, ht, plan.lmax, plan.tmax,
                        plan.npairs, omega_ready, lat->s_gf.ptr, (double *)lat->s_part.ptr, wilson_gf_blocks(lat->g),
                        d_out, out_stride, lat->stream, side, ev));
    return KLFT_OK;
  }
  for (int mu = 0; mu < nu; ++mu) {
    klft_status s = enqueue_wilson_plane(lat, plan, mu, nu, omega_ready || mu > 0, d_out + (size_t)mu * out_stride);
    if (s != KLFT_OK) return s;
  }
  return KLFT_OK;
}

// unnormalised sums over sites for a list of (Lmu, Lnu) pairs in the (mu, nu) plane
klft_status wilson_sums(klft_lattice *lat, int mu, int nu, const int *pairs, int npairs, double *sums) {
  CK(lat->s_out.ensure((size_t)(npairs > KLFT_RESULT_SLOTS ? npairs : KLFT_RESULT_SLOTS) * sizeof(double)));
  WilsonPlan plan;
  klft_status s = make_wilson_plan(lat, pairs, npairs, nu, plan);
  if (s != KLFT_OK) return s;
  s = enqueue_wilson_plane(lat, plan, mu, nu, false, (double *)lat->s_out.ptr);
  if (s != KLFT_OK) return s;
  CK(cudaMemcpyAsync(sums, lat->s_out.ptr, (size_t)npairs * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

}  // namespace klft
