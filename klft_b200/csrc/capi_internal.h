// capi_internal.h -- the lattice handle behind the C ABI and the enqueue helpers
// shared by the translation units of libklft_b200.so.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "../../include/klft_b200.h"
#include "common.cuh"
#include "kernels.cuh"

#define KLFT_RESULT_SLOTS 256

namespace klft {

// A growable device buffer owned by a handle.  With a stream attached it is
// allocated and freed stream-ordered on that stream (cudaMallocAsync /
// cudaFreeAsync), which never synchronises the device.
struct Scratch {
  void *ptr = nullptr;
  size_t cap = 0;
  cudaStream_t stream = nullptr;
  cudaError_t ensure(size_t bytes);
  void release();
};

// Pinned host result slots (KLFT_RESULT_SLOTS doubles), reused across lattices:
// cudaFreeHost would synchronise the device whenever a lattice is destroyed.
double *pinned_slots_get();
void pinned_slots_put(double *p);
// The device's default memory pool keeps freed memory for reuse (once per device).
void keep_pool_memory(int device);
// Whole-lattice host <-> device copies (hostio.cu): one DMA transfer for a
// page-locked host buffer, else chunks through the library's page-locked
// staging buffers filled and drained by host threads.  Both return after the
// host buffer may be reused (host -> device: the device copy is enqueued on st
// and complete; device -> host: the data is in dst).
cudaError_t copy_host_to_device(void *dst, const void *src, size_t bytes, cudaStream_t st);
cudaError_t copy_device_to_host(void *dst, const void *src, size_t bytes, cudaStream_t st);
// Mixed form: only the stored FP32 reals of each link cross PCIe (12 for SU(3),
// 4 for SU(2), 2 for U(1)); the host side converts from / to klft's 2 N^2
// doubles per link (lexicographic site, then direction) on the library's threads.
cudaError_t upload_links_f32(void *dst, const double *src, size_t nlinks, int nc, cudaStream_t st);
cudaError_t download_links_f32(double *dst, const void *src, size_t nlinks, int nc, cudaStream_t st);

klft_status fail(klft_status code, const char *fmt, ...);
klft_status cuda_fail(cudaError_t e, const char *what);

}  // namespace klft

namespace klft {
// The proposal arguments every sweep entry point accepts (who names the caller
// in the error message).
klft_status check_proposal(const klft_lattice *lat, double delta, int proposal, double eps, const char *who);
}  // namespace klft

struct klft_lattice {
  int nc = 0;
  int precision = 0;
  int device = 0;
  klft::Geom g{};
  uint64_t seed = 0, chain = 0;
  void *links = nullptr;
  size_t link_bytes = 0;
  cudaStream_t stream = nullptr;
  // klft_run_cycles: a second stream (created on first use) for the plaquette,
  // beside the loops' axial-gauge transformation, and for the loop kernels,
  // beside the next sweep; events: after the sweep, after the plaquette, after
  // U', after the loops
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_up = nullptr, ev_loops = nullptr;
  uint32_t *d_counters = nullptr;  // [0] sweep, [1] trajectory, [2] cycle
  double *h_results = nullptr;     // pinned, KLFT_RESULT_SLOTS doubles
  klft::Scratch s_part, s_out, s_aux, s_stage, s_wl, s_hmc, s_gf, s_tab, s_tune;
  int hmc_cap = 0;  // trajectories the HMC buffers in s_hmc are laid out for
  int hmc_generators = KLFT_GENERATORS_REFERENCE;
  klft::Defect defect{0, 1, {0, 0, 0}, 1.0, nullptr};
  std::mutex mtx;
  int dtype() const { return precision == KLFT_PRECISION_FP64 ? 0 : 1; }
};

namespace klft {
klft_status lattice_sync(klft_lattice *lat);
Geom make_geom(int ndims, const int *L);
// may_tune = false: use only tuned values already known (no timing, no scratch)
klft_status enqueue_sweeps(klft_lattice *lat, double beta, double delta, int nhits, int proposal, double eps,
                           int nsweeps, unsigned long long *d_nacc, const Defect &df, bool may_tune = true);
klft_status enqueue_plaquette(klft_lattice *lat, int slot);
double normalize_plaquette(const klft_lattice *lat, double sum);
double normalize_wilson(const klft_lattice *lat, double sum);
// One lattice's share of a multi-chain sweep (batch.cu).
struct SweepItem {
  klft_lattice *lat;
  MetroArgs a;
  Defect df;
  int acc_index;  // accept-counter index; < 0: the item's position
};
// Side streams for enqueue_multi_sweep: the chains of different launch groups
// share no data, so group g > 0 may run on side[(g - 1) % nside], forked from
// and joined back into the main stream with the given events (also inside a
// stream capture, where the fork and join become graph edges).
struct StreamFork {
  cudaEvent_t fork;
  const cudaStream_t *side;
  const cudaEvent_t *join;  // one per side stream
  int nside;
};
// block: threads per CTA of the multi-chain launches (32, 64 or 128; results do not depend on it)
klft_status enqueue_multi_sweep(const std::vector<SweepItem> &items, unsigned long long *nacc, const uint32_t *slot,
                                cudaStream_t st, int acc_stride, int *nlaunch, const StreamFork *fork = nullptr,
                                int block = 128);
// sweep counters += 1: a device array of counter pointers, or a host list
cudaError_t launch_advance_many(uint32_t *const *d_ctrs, int n, cudaStream_t st);
cudaError_t launch_advance_list(const std::vector<uint32_t *> &ctrs, cudaStream_t st, int *nlaunch);
// HMC pieces on the lattice's stream (hmc.cu).  hmc_prepare sizes every buffer
// for ntraj trajectories (it may allocate; nothing else below does).
klft_status hmc_prepare(klft_lattice *lat, int ntraj);
// trajectory k (< ntraj of hmc_prepare): momenta, H, integrate, H', accept/restore
klft_status hmc_enqueue_trajectory(klft_lattice *lat, double beta, double tau, int nsteps, int integrator, int k);
// d_out[0] = accepted trajectories, d_out[1] = sum exp(-dH), d_out[2] = sum dH over the first ntraj
klft_status hmc_enqueue_summary(klft_lattice *lat, int ntraj, double *d_out);
// device bytes of the HMC buffers for ntraj trajectories
size_t hmc_footprint(int nc, int dtype, const Geom &g, int ntraj);

// A Wilson-loop pair list: the pairs on the device (direct form, in s_tab) and
// the per-length tables the gauge-fixed kernel takes in its parameters.
struct WilsonPlan {
  int npairs = 0, lmax = 0, tmax = 0;
  bool gf = false;
  size_t tab_off = 0;  // the pairs' position (ints) in the handle's device table
  // gauge-fixed form: loops of length L are entries off[L] .. off[L+1]-1 of (T, pair)
  std::vector<int> off, T, p;
};
// tab_off: where the pairs go in lat->s_tab (several plans in flight at once
// use disjoint ranges; the caller then sizes s_tab for all of them first)
// nplanes: the planes one enqueue_wilson_spatial call covers (scratch for one U' each)
klft_status make_wilson_plan(klft_lattice *lat, const int *pairs, int npairs, int nu, WilsonPlan &plan,
                             size_t tab_off = 0, int nplanes = 1);
klft_status enqueue_wilson_plane(klft_lattice *lat, const WilsonPlan &plan, int mu, int nu, bool omega_ready,
                                 double *d_out);
// side / ev: the gauge-fixed form's loop kernels on side after ev (see launch_wilson_gf)
klft_status enqueue_wilson_spatial(klft_lattice *lat, const WilsonPlan &plan, bool omega_ready, double *d_out,
                                   int out_stride, cudaStream_t side = nullptr, cudaEvent_t ev = nullptr);
klft_status wilson_sums(klft_lattice *lat, int mu, int nu, const int *pairs, int npairs, double *sums);
}  // namespace klft
