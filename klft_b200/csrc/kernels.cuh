// kernels.cuh -- host-side launch interface of the device kernels.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace klft {

struct MetroArgs {
  double beta, delta, eps;
  int nhits, proposal;
  uint64_t seed, chain;
  const double *bm = nullptr;  // FP64 Box-Muller table (bm_table()), set at launch
};

// The FP64 Box-Muller table of the current device (BM_TAB radii, then BM_TAB
// (cos, sin) pairs, 1.5 MB), built on the host and uploaded on first use; call
// it outside stream capture (lattice creation does).  Null on a CUDA error.
const double *bm_table();

// Launches per sweep: 2 Nd link passes for the SU(3) exp(i eps H) proposal
// (proposal 1), else the reference's 2^Nd site classes.
KLFT_HD int metropolis_passes(int nc, int proposal, int nd) { return nc == 3 && proposal == 1 ? 2 * nd : 1 << nd; }

// dtype: 0 = double (plain FP64 form), 1 = float (mixed form)
// val: the site class, or the link pass 2 mu + parity of the exp proposal
cudaError_t launch_metropolis_pass(int nc, int dtype, void *links, const Geom &g, int val, const MetroArgs &a,
                                   const uint32_t *d_sweep, unsigned long long *d_nacc, const Defect &df, int block,
                                   cudaStream_t st);
cudaError_t launch_advance(uint32_t *d_counter, cudaStream_t st);

cudaError_t launch_init(int nc, int dtype, void *links, const Geom &g, int hot, uint64_t seed, uint64_t chain,
                        cudaStream_t st);
// host AoS FP64 staging buffer <-> device layout
cudaError_t launch_import(int nc, int dtype, void *links, const Geom &g, const double *aos, cudaStream_t st);
cudaError_t launch_export(int nc, int dtype, const void *links, const Geom &g, double *aos, cudaStream_t st);
// mixed form: the stored FP32 reals per link in interchange order (see field.cu)
cudaError_t launch_import_f32(int nc, void *links, const Geom &g, const float *aos, cudaStream_t st);
cudaError_t launch_export_f32(int nc, const void *links, const Geom &g, float *aos, cudaStream_t st);
// zero the links across the open boundary (no-op when periodic)
cudaError_t launch_open_boundary(int nc, int dtype, void *links, const Geom &g, cudaStream_t st);
cudaError_t launch_reunitarize(int nc, int dtype, void *links, const Geom &g, cudaStream_t st);
// max ||U^dagger U - 1||_F -> *d_out (via partials)
cudaError_t launch_unitarity(int nc, int dtype, const void *links, const Geom &g, double *d_part, double *d_out,
                             cudaStream_t st);
// staples of every link, written in host AoS FP64 layout
cudaError_t launch_staple_field(int nc, int dtype, const void *links, const Geom &g, double *aos, cudaStream_t st);

// sum over sites of sum_{mu<nu<nu_end} Re Tr P_{mu nu} (nu_end < 0: all planes), unnormalised, into *d_out;
// f64_terms: every product term summed in FP64 (else each plane's trace in the link precision)
cudaError_t launch_plaquette(int nc, int dtype, const void *links, const Geom &g, double *d_part, int nblk,
                             double *d_out, cudaStream_t st, int nu_end = -1, bool f64_terms = false);
// Wilson loops of a pair list in the (mu, nu) plane; d_out[k] = sum over sites Re Tr W
cudaError_t launch_wilson_direct(int nc, int dtype, const void *links, const Geom &g, int mu, int nu,
                                 const int *d_pairs, int npairs, double *d_part, int nblk, double *d_out,
                                 cudaStream_t st);

// Wilson loops of a pair list in the (mu, nu) plane by axial gauge fixing (wilson.cu)
// scratch of the gauge-fixed loops of nplanes planes sharing nu (one Omega, one U' per plane)
size_t wilson_gf_scratch(int nc, int dtype, const Geom &g, int nu, int tmax, int nplanes = 1);
size_t wilson_gf_smem(int nc, int dtype, const Geom &g, int nu, int tmax, int npairs);
int wilson_gf_blocks(const Geom &g);
// h_tab = {off[lmax+2], T[npairs], p[npairs]} on the host (passed in the kernel
// parameters); npairs, lmax <= WL_MAXP
constexpr int WL_MAXP = 128;
// Loops of the planes (mus[i], nu), i < nplanes <= 3, sharing one axial-gauge
// transformation; plane i's sums go to d_out[i * out_stride + k]; d_part holds
// nblk * npairs * nplanes doubles.  With st_loops, the loop kernels and the
// reduction run there after an event (ev, recorded on st once U' is written):
// only Omega and U' read the links, so st may go on to change them.
cudaError_t launch_wilson_gf(int nc, int dtype, const void *links, const Geom &g, const int *mus, int nplanes,
                             int nu, const int *const *h_tab, int lmax, int tmax, int npairs, bool omega_ready,
                             void *scratch, double *d_part, int nblk, double *d_out, int out_stride,
                             cudaStream_t st, cudaStream_t st_loops = nullptr, cudaEvent_t ev = nullptr);

int plaquette_blocks(const Geom &g);
// ordered final reduction of nblk partials for each of n outputs
cudaError_t launch_reduce_partials(const double *d_part, int nblk, int n, double *d_out, cudaStream_t st);

}  // namespace klft
