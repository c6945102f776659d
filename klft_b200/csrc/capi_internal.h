// capi_internal.h -- the lattice handle behind the C ABI and the enqueue helpers
// shared by the translation units of libklft_b200.so.
#pragma once
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/klft_b200.h"
#include "common.cuh"

#define KLFT_RESULT_SLOTS 256

namespace klft {

// A growable device buffer owned by a handle.
struct Scratch {
  void *ptr = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes);
  void release();
};

klft_status fail(klft_status code, const char *fmt, ...);
klft_status cuda_fail(cudaError_t e, const char *what);

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
  uint32_t *d_counters = nullptr;  // [0] sweep, [1] trajectory, [2] cycle
  double *h_results = nullptr;     // pinned, KLFT_RESULT_SLOTS doubles
  klft::Scratch s_part, s_out, s_aux, s_stage, s_wl, s_hmc, s_gf, s_tab, s_tune;
  klft::Defect defect{0, 1, {0, 0, 0}, 1.0, nullptr};
  std::mutex mtx;
  int dtype() const { return precision == KLFT_PRECISION_FP64 ? 0 : 1; }
};

namespace klft {
klft_status lattice_sync(klft_lattice *lat);
// may_tune = false: use only tuned values already known (no timing, no scratch)
klft_status enqueue_sweeps(klft_lattice *lat, double beta, double delta, int nhits, int proposal, double eps,
                           int nsweeps, unsigned long long *d_nacc, const Defect &df, bool may_tune = true);
klft_status enqueue_plaquette(klft_lattice *lat, int slot);
double normalize_plaquette(const klft_lattice *lat, double sum);
double normalize_wilson(const klft_lattice *lat, double sum);
// Device tables of a Wilson-loop pair list (offsets are int indices into s_tab).
struct WilsonPlan {
  int npairs = 0, lmax = 0, tmax = 0;
  bool gf = false;
  int off_at = 0, t_at = 0, p_at = 0;
};
klft_status make_wilson_plan(klft_lattice *lat, const int *pairs, int npairs, int nu, WilsonPlan &plan);
klft_status enqueue_wilson_plane(klft_lattice *lat, const WilsonPlan &plan, int mu, int nu, bool omega_ready,
                                 double *d_out);
klft_status wilson_sums(klft_lattice *lat, int mu, int nu, const int *pairs, int npairs, double *sums);
}  // namespace klft
