// hmc.cu -- Hybrid Monte Carlo for U(1), SU(2), SU(3) gauge fields.
//
// Semantics restate the reference's (non-building) HMC stack:
//   HMC::hmc_step                      HMC.hpp:48-71
//   Leapfrog::integrate                Integrator.hpp:22-54 (n_steps + 1 gauge updates)
//   GaugeMonomial derivative / H       GaugeMonomial.hpp:19-37
//   update_momentum / update_gauge /
//   kinetic_energy / randomize_momentum HamiltonianField.hpp:23-59
//   Adjoint / exp                       AdjointGroup.hpp:13-19, 98-105, 114-117, 170-173
// with the Lie-algebra conventions of the reference extended to SU(3) through
// the Gell-Mann generators: U <- exp(i dt sum_a p_a t_a) U, H = sum p^2 / 2 -
// (beta/Nc) sum_P Re Tr P, F_a = (beta/Nc) Im Tr(t_a U S) with S the staple.
//
// Momenta are structure of arrays, P[(mu*ncomp + a)*V + lin(x)], in the link
// precision (FP32 in the mixed form); energies and dH are FP64 reductions; the
// accept/reject and the restore of rejected links run on the device, so a
// trajectory is one stream of launches with no host round trip.
#include "../../include/klft_b200.h"
#include "capi_internal.h"
#include "group.cuh"
#include "kernels.cuh"
#include "staple.cuh"

namespace klft {

constexpr int HMC_THREADS = 256;

template <int NC, typename T>
__global__ void __launch_bounds__(HMC_THREADS) momenta_kernel(T *P, Geom g, uint64_t seed, uint64_t chain,
                                                              const uint32_t *__restrict__ ctr) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const int mu = (int)(t / g.V);
  const long long lin = t - (long long)mu * g.V;
  const Site x = site_from_lin(g, lin);
  constexpr int nc = Alg<NC>::n;
  Stream st(seed, chain, site_lex(g, x), ctr[1], KIND_MOMENTUM, (uint32_t)mu);
  double gs[8];
#pragma unroll
  for (int k = 0; k < (nc + 1) / 2; ++k) st.gauss2(gs[2 * k], gs[2 * k + 1]);
#pragma unroll
  for (int a = 0; a < nc; ++a) P[((long long)mu * nc + a) * g.V + lin] = (T)gs[a];
}

// P -= dt * (beta/Nc) Adj(U S): the force of GaugeMonomial::derivative fused with
// HamiltonianField::update_momentum; one thread per link.
// Grid: x over the links of one direction, y = mu (so mu is uniform per CTA and
// the staple's site arithmetic is compiled per direction).
template <int NC, int ND, typename T>
__global__ void __launch_bounds__(128) force_update_kernel(Links<NC, T> U, T *P, Geom g, T bnc, T dt) {
  const long long lin = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (lin >= g.V) return;
  const int mu = (int)blockIdx.y;
  const Site x = g.Vh < (1LL << 31) ? site_from_lin32(g, (unsigned)lin) : site_from_lin(g, lin);
  Mat<NC, T> S;
  if constexpr (NC == 3) {
    // SU(3): the rolled staple (the unrolled products cost occupancy: 150 registers)
    const Defect none{0, 1, {0, 0, 0}, 1.0, nullptr};
    S = staple<NC, ND, T>(U, g, x, mu, none);
  } else {
    S = staple_dispatch<NC, ND, T>(U, g, x, mu);
  }
  const Mat<NC, T> M = mul(U.load(lin, mu), S);
  constexpr int nc = Alg<NC>::n;
  T v[nc];
  adjoint(M, v);
#pragma unroll
  for (int a = 0; a < nc; ++a) {
    T &p = P[((long long)mu * nc + a) * g.V + lin];
    p -= dt * (bnc * v[a]);
  }
}

// U <- exp(dt P) U (HamiltonianField::update_gauge); one thread per link.
template <int NC, typename T>
__global__ void __launch_bounds__(HMC_THREADS) gauge_update_kernel(Links<NC, T> U, const T *P, Geom g, T dt) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const int mu = (int)(t / g.V);
  const long long lin = t - (long long)mu * g.V;
  constexpr int nc = Alg<NC>::n;
  T p[nc];
#pragma unroll
  for (int a = 0; a < nc; ++a) p[a] = P[((long long)mu * nc + a) * g.V + lin];
  U.store(lin, mu, mul(expmap(p, dt, (const Mat<NC, T> *)nullptr), U.load(lin, mu)));
}

// sum of p^2 / 2 over the field, FP64, block partials
template <typename T>
__global__ void __launch_bounds__(HMC_THREADS) kinetic_kernel(const T *P, long long n, double *part) {
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * HMC_THREADS + threadIdx.x; i < n; i += (long long)gridDim.x * HMC_THREADS) {
    const double p = (double)P[i];
    acc += 0.5 * p * p;
  }
  __shared__ double red[HMC_THREADS / 32];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < HMC_THREADS / 32; ++w) s += red[w];
    part[blockIdx.x] = s;
  }
}

// slots: [0] K_old [1] plaquette sum old [2] K_new [3] plaquette sum new
// HMC.hpp:58-68: dH = (K_new - K_old) + (H_gauge_new - H_gauge_old); reject when
// dH > 0 and u > exp(-dH).  Writes dH and the decision, advances the trajectory
// counter.
__global__ void hmc_accept_kernel(const double *slots, double bnc, uint64_t seed, uint64_t chain, uint32_t *ctr,
                                  double *dH_out, int *acc_out) {
  const double g_old = -bnc * slots[1], g_new = -bnc * slots[3];
  double dH = 0.0;
  dH += slots[2] - slots[0];
  dH += g_new - g_old;
  int accept = 1;
  if (dH > 0.0) {
    Stream st(seed, chain, 0u, ctr[1], KIND_HMC_ACCEPT, 0u);
    if (st.next() > exp(-dH)) accept = 0;
  }
  *dH_out = dH;
  *acc_out = accept;
  ctr[1] += 1u;
}

// restore the saved links of a rejected trajectory
__global__ void restore_if_rejected_kernel(uint4 *links, const uint4 *saved, long long n16, const int *accepted) {
  if (*accepted) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (long long)gridDim.x * blockDim.x)
    links[i] = saved[i];
}

// ------------------------------------------------------------------ launch helpers
static unsigned grid_for(long long n, int b) { return (unsigned)((n + b - 1) / b); }

#define KLFT_HMC_DISPATCH(nc, dtype, CALL)                                    \
  do {                                                                        \
    if (dtype == 0) {                                                         \
      using T = double;                                                       \
      if (nc == 1) { constexpr int NC = 1; CALL; }                            \
      else if (nc == 2) { constexpr int NC = 2; CALL; }                       \
      else { constexpr int NC = 3; CALL; }                                    \
    } else {                                                                  \
      using T = float;                                                        \
      if (nc == 1) { constexpr int NC = 1; CALL; }                            \
      else if (nc == 2) { constexpr int NC = 2; CALL; }                       \
      else { constexpr int NC = 3; CALL; }                                    \
    }                                                                         \
  } while (0)

static int ncomp_of(int nc) { return nc == 1 ? 1 : (nc == 2 ? 3 : 8); }

cudaError_t launch_momenta(const klft_lattice *lat, void *P) {
  const Geom &g = lat->g;
  KLFT_HMC_DISPATCH(lat->nc, lat->dtype(),
                    (momenta_kernel<NC, T><<<grid_for(g.V * g.nd, HMC_THREADS), HMC_THREADS, 0, lat->stream>>>(
                        (T *)P, g, lat->seed, lat->chain, lat->d_counters)));
  return cudaGetLastError();
}

cudaError_t launch_force_update(const klft_lattice *lat, void *P, double beta, double dt) {
  const Geom &g = lat->g;
#define KLFT_FU(NDV)                                                                                        \
  force_update_kernel<NC, NDV, T><<<dim3(grid_for(g.V, 128), NDV), 128, 0, lat->stream>>>(                   \
      Links<NC, T>{(cx<T> *)lat->links, g.V}, (T *)P, g, (T)(beta / (double)NC), (T)dt)
  KLFT_HMC_DISPATCH(lat->nc, lat->dtype(), ({
    if (g.nd == 2) KLFT_FU(2);
    else if (g.nd == 3) KLFT_FU(3);
    else KLFT_FU(4);
  }));
#undef KLFT_FU
  return cudaGetLastError();
}

cudaError_t launch_gauge_update(const klft_lattice *lat, const void *P, double dt) {
  const Geom &g = lat->g;
  KLFT_HMC_DISPATCH(lat->nc, lat->dtype(),
                    (gauge_update_kernel<NC, T><<<grid_for(g.V * g.nd, HMC_THREADS), HMC_THREADS, 0, lat->stream>>>(
                        Links<NC, T>{(cx<T> *)lat->links, g.V}, (const T *)P, g, (T)dt)));
  return cudaGetLastError();
}

cudaError_t launch_kinetic(const klft_lattice *lat, const void *P, double *d_part, int nblk, double *d_out) {
  const long long n = lat->g.V * lat->g.nd * ncomp_of(lat->nc);
  if (lat->dtype() == 0)
    kinetic_kernel<double><<<nblk, HMC_THREADS, 0, lat->stream>>>((const double *)P, n, d_part);
  else
    kinetic_kernel<float><<<nblk, HMC_THREADS, 0, lat->stream>>>((const float *)P, n, d_part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_reduce_partials(d_part, nblk, 1, d_out, lat->stream);
}

}  // namespace klft

// ------------------------------------------------------------------ C ABI
using namespace klft;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

namespace {

// HMC scratch in lat->s_hmc: [P][saved links][slots 8 doubles][dH ntraj][acc ntraj]
struct HmcBufs {
  void *P;
  void *saved;
  double *slots;
  double *dH;
  int *acc;
};

size_t p_bytes(const klft_lattice *lat) {
  return (size_t)lat->g.V * lat->g.nd * ncomp_of(lat->nc) * (lat->dtype() == 0 ? 8 : 4);
}

// The layout depends on the trajectory capacity kept in the handle, which only
// grows, so buffers sized once for ntraj keep their places for every k < ntraj.
klft_status hmc_bufs(klft_lattice *lat, int ntraj, HmcBufs &b) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  if (ntraj < lat->hmc_cap) ntraj = lat->hmc_cap;
  const size_t pb = al(p_bytes(lat)), lb = al(lat->link_bytes);
  const size_t need = pb + lb + al(8 * sizeof(double)) + al((size_t)ntraj * sizeof(double)) + al((size_t)ntraj * sizeof(int));
  CK(lat->s_hmc.ensure(need));
  lat->hmc_cap = ntraj;
  char *base = (char *)lat->s_hmc.ptr;
  b.P = base;
  b.saved = base + pb;
  b.slots = (double *)(base + pb + lb);
  b.dH = (double *)(base + pb + lb + al(8 * sizeof(double)));
  b.acc = (int *)(base + pb + lb + al(8 * sizeof(double)) + al((size_t)ntraj * sizeof(double)));
  const int nblk = plaquette_blocks(lat->g);
  CK(lat->s_part.ensure((size_t)nblk * sizeof(double)));
  return KLFT_OK;
}

klft_status enqueue_energies(klft_lattice *lat, const HmcBufs &b, double *slot_k, double *slot_p) {
  const int nblk = plaquette_blocks(lat->g);
  CK(launch_kinetic(lat, b.P, (double *)lat->s_part.ptr, nblk, slot_k));
  CK(launch_plaquette(lat->nc, lat->dtype(), lat->links, lat->g, (double *)lat->s_part.ptr, nblk, slot_p,
                      lat->stream, -1, true));
  return KLFT_OK;
}

// Integrator.hpp:26-53 (reference leapfrog), the standard leapfrog, and the
// 2nd-order minimum-norm (Omelyan) scheme; then reunitarisation.
// With t_a / 2 generators a step of length dt moves the links and momenta
// exactly as a reference step of length dt / 2 (the force halves and the
// exponent halves), so the HALF normalisation integrates tau / 2.
klft_status enqueue_integrate(klft_lattice *lat, const HmcBufs &b, double beta, double tau, int nsteps,
                              int integrator) {
  const double dt = (lat->hmc_generators == KLFT_GENERATORS_HALF ? 0.5 : 1.0) * tau / (double)nsteps;
  auto P = [&](double h) -> klft_status {
    CK(launch_force_update(lat, b.P, beta, h));
    return KLFT_OK;
  };
  auto U = [&](double h) -> klft_status {
    CK(launch_gauge_update(lat, b.P, h));
    return KLFT_OK;
  };
  klft_status s = KLFT_OK;
#define STEP(x) \
  if ((s = (x)) != KLFT_OK) return s
  if (integrator == KLFT_INTEGRATOR_REFERENCE_LEAPFROG) {
    STEP(P(dt / 2.0));
    STEP(U(dt));
    for (int i = 0; i < nsteps; ++i) {
      STEP(P(dt));
      STEP(U(dt));
    }
    STEP(P(dt / 2.0));
  } else if (integrator == KLFT_INTEGRATOR_LEAPFROG) {
    STEP(P(dt / 2.0));
    for (int i = 0; i < nsteps; ++i) {
      STEP(U(dt));
      STEP(P(i == nsteps - 1 ? dt / 2.0 : dt));
    }
  } else {
    const double lam = 0.1931833275037836;
    for (int i = 0; i < nsteps; ++i) {
      STEP(P(lam * dt));
      STEP(U(dt / 2.0));
      STEP(P((1.0 - 2.0 * lam) * dt));
      STEP(U(dt / 2.0));
      STEP(P(lam * dt));
    }
  }
#undef STEP
  CK(launch_reunitarize(lat->nc, lat->dtype(), lat->links, lat->g, lat->stream));
  return KLFT_OK;
}

klft_status check_hmc_args(klft_lattice *lat, double tau, int nsteps, int integrator, const char *who) {
  if (!lat) return fail(KLFT_EINVAL, "%s: null handle", who);
  if (nsteps < 1) return fail(KLFT_EINVAL, "%s: n_steps must be >= 1", who);
  if (!(tau == tau)) return fail(KLFT_EINVAL, "%s: NaN tau", who);
  if (integrator < KLFT_INTEGRATOR_REFERENCE_LEAPFROG || integrator > KLFT_INTEGRATOR_OMELYAN)
    return fail(KLFT_EINVAL, "%s: unknown integrator %d", who, integrator);
  return KLFT_OK;
}

// host layout P[(site*Nd + mu)*ncomp + a] (double) <-> device SoA in the link precision
template <typename T>
__global__ void p_import_kernel(T *P, Geom g, int ncomp, const double *h) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const long long lex = t / g.nd;
  const int mu = (int)(t - lex * g.nd);
  const long long lin = site_lin(g, site_from_lex(g, lex));
  for (int a = 0; a < ncomp; ++a) P[((long long)mu * ncomp + a) * g.V + lin] = (T)h[t * ncomp + a];
}
template <typename T>
__global__ void p_export_kernel(const T *P, Geom g, int ncomp, double *h) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const long long lex = t / g.nd;
  const int mu = (int)(t - lex * g.nd);
  const long long lin = site_lin(g, site_from_lex(g, lex));
  for (int a = 0; a < ncomp; ++a) h[t * ncomp + a] = (double)P[((long long)mu * ncomp + a) * g.V + lin];
}

__global__ void hmc_summary_kernel(const double *dH, const int *acc, int n, double *out) {
  double a = 0.0, e = 0.0, d = 0.0;
  for (int k = 0; k < n; ++k) {
    a += acc[k] ? 1.0 : 0.0;
    e += exp(-dH[k]);
    d += dH[k];
  }
  out[0] = a;
  out[1] = e;
  out[2] = d;
}

}  // namespace

namespace klft {

size_t hmc_footprint(int nc, int dtype, const Geom &g, int ntraj) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t pb = (size_t)g.V * g.nd * ncomp_of(nc) * (dtype == 0 ? 8 : 4);
  const size_t lb = (size_t)g.V * g.nd * link_planes(nc, dtype) * (dtype == 0 ? 16 : 8);
  return al(pb) + al(lb) + al(8 * sizeof(double)) + al((size_t)ntraj * sizeof(double)) +
         al((size_t)ntraj * sizeof(int)) + (size_t)plaquette_blocks(g) * sizeof(double);
}

klft_status hmc_prepare(klft_lattice *lat, int ntraj) {
  HmcBufs b;
  return hmc_bufs(lat, ntraj < 1 ? 1 : ntraj, b);
}

klft_status hmc_enqueue_trajectory(klft_lattice *lat, double beta, double tau, int nsteps, int integrator, int k) {
  HmcBufs b;
  klft_status s = hmc_bufs(lat, k + 1, b);
  if (s != KLFT_OK) return s;
  CK(launch_momenta(lat, b.P));
  if ((s = enqueue_energies(lat, b, b.slots + 0, b.slots + 1)) != KLFT_OK) return s;
  CK(cudaMemcpyAsync(b.saved, lat->links, lat->link_bytes, cudaMemcpyDeviceToDevice, lat->stream));
  if ((s = enqueue_integrate(lat, b, beta, tau, nsteps, integrator)) != KLFT_OK) return s;
  if ((s = enqueue_energies(lat, b, b.slots + 2, b.slots + 3)) != KLFT_OK) return s;
  hmc_accept_kernel<<<1, 1, 0, lat->stream>>>(b.slots, beta / (double)lat->nc, lat->seed, lat->chain,
                                              lat->d_counters, b.dH + k, b.acc + k);
  CK(cudaGetLastError());
  restore_if_rejected_kernel<<<296, 256, 0, lat->stream>>>((uint4 *)lat->links, (const uint4 *)b.saved,
                                                           (long long)(lat->link_bytes / 16), b.acc + k);
  CK(cudaGetLastError());
  return KLFT_OK;
}

klft_status hmc_enqueue_summary(klft_lattice *lat, int ntraj, double *d_out) {
  HmcBufs b;
  klft_status s = hmc_bufs(lat, ntraj < 1 ? 1 : ntraj, b);
  if (s != KLFT_OK) return s;
  hmc_summary_kernel<<<1, 1, 0, lat->stream>>>(b.dH, b.acc, ntraj, d_out);
  CK(cudaGetLastError());
  return KLFT_OK;
}

}  // namespace klft

extern "C" {

klft_status klft_hmc_set_momenta(klft_lattice *lat, const double *host) {
  if (!lat || !host) return fail(KLFT_EINVAL, "klft_hmc_set_momenta: null pointer");
  std::lock_guard<std::mutex> guard(lat->mtx);
  HmcBufs b;
  klft_status s = hmc_bufs(lat, 1, b);
  if (s != KLFT_OK) return s;
  const size_t n = (size_t)lat->g.V * lat->g.nd * ncomp_of(lat->nc);
  CK(lat->s_stage.ensure(n * sizeof(double)));
  CK(cudaMemcpyAsync(lat->s_stage.ptr, host, n * sizeof(double), cudaMemcpyHostToDevice, lat->stream));
  const unsigned grid = grid_for(lat->g.V * lat->g.nd, 256);
  if (lat->dtype() == 0)
    p_import_kernel<double><<<grid, 256, 0, lat->stream>>>((double *)b.P, lat->g, ncomp_of(lat->nc),
                                                             (const double *)lat->s_stage.ptr);
  else
    p_import_kernel<float><<<grid, 256, 0, lat->stream>>>((float *)b.P, lat->g, ncomp_of(lat->nc),
                                                            (const double *)lat->s_stage.ptr);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_hmc_get_momenta(klft_lattice *lat, double *host) {
  if (!lat || !host) return fail(KLFT_EINVAL, "klft_hmc_get_momenta: null pointer");
  std::lock_guard<std::mutex> guard(lat->mtx);
  HmcBufs b;
  klft_status s = hmc_bufs(lat, 1, b);
  if (s != KLFT_OK) return s;
  const size_t n = (size_t)lat->g.V * lat->g.nd * ncomp_of(lat->nc);
  CK(lat->s_stage.ensure(n * sizeof(double)));
  const unsigned grid = grid_for(lat->g.V * lat->g.nd, 256);
  if (lat->dtype() == 0)
    p_export_kernel<double><<<grid, 256, 0, lat->stream>>>((const double *)b.P, lat->g, ncomp_of(lat->nc),
                                                             (double *)lat->s_stage.ptr);
  else
    p_export_kernel<float><<<grid, 256, 0, lat->stream>>>((const float *)b.P, lat->g, ncomp_of(lat->nc),
                                                            (double *)lat->s_stage.ptr);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, lat->s_stage.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_hmc_refresh_momenta(klft_lattice *lat) {
  if (!lat) return fail(KLFT_EINVAL, "klft_hmc_refresh_momenta: null handle");
  std::lock_guard<std::mutex> guard(lat->mtx);
  HmcBufs b;
  klft_status s = hmc_bufs(lat, 1, b);
  if (s != KLFT_OK) return s;
  CK(launch_momenta(lat, b.P));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_gauge_force(klft_lattice *lat, double beta, double *host_force) {
  if (!lat || !host_force) return fail(KLFT_EINVAL, "klft_gauge_force: null pointer");
  // F = (P_before - P_after) with a unit step from P = 0: F = (beta/Nc) Adj(U S)
  std::lock_guard<std::mutex> guard(lat->mtx);
  HmcBufs b;
  klft_status s = hmc_bufs(lat, 1, b);
  if (s != KLFT_OK) return s;
  CK(cudaMemsetAsync(b.P, 0, p_bytes(lat), lat->stream));
  CK(launch_force_update(lat, b.P, beta, lat->hmc_generators == KLFT_GENERATORS_HALF ? -0.5 : -1.0));
  const size_t n = (size_t)lat->g.V * lat->g.nd * ncomp_of(lat->nc);
  CK(lat->s_stage.ensure(n * sizeof(double)));
  const unsigned grid = grid_for(lat->g.V * lat->g.nd, 256);
  if (lat->dtype() == 0)
    p_export_kernel<double><<<grid, 256, 0, lat->stream>>>((const double *)b.P, lat->g, ncomp_of(lat->nc),
                                                             (double *)lat->s_stage.ptr);
  else
    p_export_kernel<float><<<grid, 256, 0, lat->stream>>>((const float *)b.P, lat->g, ncomp_of(lat->nc),
                                                            (double *)lat->s_stage.ptr);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host_force, lat->s_stage.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_hmc_energies(klft_lattice *lat, double beta, double *kinetic, double *gauge_action) {
  if (!lat) return fail(KLFT_EINVAL, "klft_hmc_energies: null handle");
  std::lock_guard<std::mutex> guard(lat->mtx);
  HmcBufs b;
  klft_status s = hmc_bufs(lat, 1, b);
  if (s != KLFT_OK) return s;
  s = enqueue_energies(lat, b, b.slots, b.slots + 1);
  if (s != KLFT_OK) return s;
  double h[2];
  CK(cudaMemcpyAsync(h, b.slots, sizeof h, cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  if (kinetic) *kinetic = h[0];
  if (gauge_action) *gauge_action = -(beta / (double)lat->nc) * h[1];
  return KLFT_OK;
}

klft_status klft_hmc_set_generators(klft_lattice *lat, int generators) {
  if (!lat) return fail(KLFT_EINVAL, "klft_hmc_set_generators: null handle");
  if (generators != KLFT_GENERATORS_REFERENCE && generators != KLFT_GENERATORS_HALF)
    return fail(KLFT_EINVAL, "klft_hmc_set_generators: unknown normalisation %d", generators);
  std::lock_guard<std::mutex> guard(lat->mtx);
  lat->hmc_generators = generators;
  return KLFT_OK;
}

klft_status klft_hmc_integrate(klft_lattice *lat, double beta, double tau, int nsteps, int integrator) {
  klft_status s = check_hmc_args(lat, tau, nsteps, integrator, "klft_hmc_integrate");
  if (s != KLFT_OK) return s;
  std::lock_guard<std::mutex> guard(lat->mtx);
  HmcBufs b;
  if ((s = hmc_bufs(lat, 1, b)) != KLFT_OK) return s;
  if ((s = enqueue_integrate(lat, b, beta, tau, nsteps, integrator)) != KLFT_OK) return s;
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_hmc_trajectories(klft_lattice *lat, double beta, double tau, int nsteps, int integrator, int ntraj,
                                  double *dH_out, int *accepted_out) {
  klft_status s = check_hmc_args(lat, tau, nsteps, integrator, "klft_hmc_trajectories");
  if (s != KLFT_OK) return s;
  if (ntraj < 0) return fail(KLFT_EINVAL, "klft_hmc_trajectories: negative count");
  if (ntraj == 0) return KLFT_OK;
  std::lock_guard<std::mutex> guard(lat->mtx);
  HmcBufs b;
  if ((s = hmc_bufs(lat, ntraj, b)) != KLFT_OK) return s;
  for (int k = 0; k < ntraj; ++k)
    if ((s = hmc_enqueue_trajectory(lat, beta, tau, nsteps, integrator, k)) != KLFT_OK) return s;
  if (dH_out) CK(cudaMemcpyAsync(dH_out, b.dH, (size_t)ntraj * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  if (accepted_out)
    CK(cudaMemcpyAsync(accepted_out, b.acc, (size_t)ntraj * sizeof(int), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

}  // extern "C"
