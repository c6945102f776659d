// ptbc.cu -- parallel tempering on boundary conditions (PTBC).
//
// The reference defines the defect (PTBCGaugeField.hpp:30-36, set_defect
// :187-198, shift_defect :200-206, accessors :209-229): links mu = 0 at x0 = 0
// whose spatial coordinates lie in pos + [0, len) (periodic) are multiplied by
// c_r, so a plaquette carries weight c_r^n with n in {0, 1, 2} its number of
// defect links.  The sweep kernels take the defect as a `Defect` argument (the
// staple and dS see the weighted links).  The reference has no replica swap;
// this file adds it:
//   S_r(U) = S_bulk(U) + sum_P (c_r^n(P) - 1) s_P(U),  s_P = -(beta/Nc) Re Tr U_P,
// and swapping the coefficients c_k, c_{k+1} held by lattices a, b changes the
// total action by
//   dS = sum_{n=1,2} (c_k^n - c_{k+1}^n) (A_n(b) - A_n(a)),
//   A_n(X) = sum over the plaquettes of X with n defect links of s_P.
// Only defect plaquettes enter, so a swap needs one small FP64 reduction per
// replica (len^(Nd-1) sites at x0 = 0).
#include <cmath>
#include <vector>

#include <cstring>
#include <vector>

#include "../../include/klft_b200.h"
#include "capi_internal.h"
#include "kernels.cuh"

namespace klft {

// Block b's partials of A_1, A_2 of one lattice (256 threads over the sites
// with x0 = 0, raw links); thread 0 writes out[0], out[1].
template <int NC, int ND, typename T>
KLFT_D void defect_partial(const Links<NC, T> &U, const Geom &g, const Defect &df, double bnc, long long b,
                           double *out) {
  long long t = b * 256 + threadIdx.x;
  const long long nsp = g.V / g.L[0];
  double a1 = 0.0, a2 = 0.0;
  if (t < nsp) {
    // spatial coordinates x1.. of this thread, x0 = 0
    Site x;
    x.set_b(0, 0);
    x.set_h(0, 0);
    long long r = t;
#pragma unroll
    for (int d = 1; d < 4; ++d) {
      const int xd = (int)(r % g.L[d]);
      r /= g.L[d];
      x.set_b(d, xd & 1);
      x.set_h(d, xd >> 1);
    }
    const bool here = in_defect(g, df, x, 0);
    const Mat<NC, T> u0 = U.load(site_lin(g, x), 0);
    const Site xp0 = site_up(g, x, 0);
#pragma unroll
    for (int i = 1; i < ND; ++i) {
      const Site xpi = site_up(g, x, i);
      const int n = (here ? 1 : 0) + (in_defect(g, df, xpi, 0) ? 1 : 0);
      if (n == 0) continue;
      // GaugePlaquette.hpp:63-79 for the (0, i) plaquette at x
      const Mat<NC, T> lmu = mul(u0, U.load(site_lin(g, xp0), i));
      const Mat<NC, T> lnu = mul(U.load(site_lin(g, x), i), U.load(site_lin(g, xpi), 0));
      const double s = -bnc * retr_nd<NC, T, double>(lmu, lnu);
      if (n == 1) a1 += s; else a2 += s;
    }
  }
  __shared__ double r1[256], r2[256];
  r1[threadIdx.x] = a1;
  r2[threadIdx.x] = a2;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      r1[threadIdx.x] += r1[threadIdx.x + s];
      r2[threadIdx.x] += r2[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = r1[0];
    out[1] = r2[0];
  }
}

template <int NC, int ND, typename T>
__global__ void __launch_bounds__(256) defect_sums_kernel(Links<NC, T> U, Geom g, Defect df, double bnc,
                                                          double *out) {
  defect_partial<NC, ND, T>(U, g, df, bnc, blockIdx.x, out + 2 * blockIdx.x);
}

// A_1, A_2 of up to 64 replicas of one (Nc, Nd, precision) in one launch:
// replica k owns CTAs [block_begin, block_begin + nblk) and partial pairs
// [part_begin, part_begin + nblk); multi_defect_reduce_kernel adds them in the
// single-lattice order into A[2 rep], A[2 rep + 1], so a replica's sums in a
// batch are bit-identical to klft_ptbc_defect_sums.
struct DefectDesc {
  void *links;
  Geom g;
  Defect df;
  int rep;
  int block_begin;
  int nblk;
  int part_begin;
};

struct DefectTable {
  int n;
  DefectDesc c[64];
};

template <int NC, int ND, typename T>
__global__ void __launch_bounds__(256) multi_defect_sums_kernel(const __grid_constant__ DefectTable tab, double bnc,
                                                                double *part) {
  int lo = 0, hi = tab.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tab.c[mid].block_begin <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const DefectDesc &c = tab.c[lo];
  const int b = (int)blockIdx.x - c.block_begin;
  defect_partial<NC, ND, T>(Links<NC, T>{(cx<T> *)c.links, c.g.V}, c.g, c.df, bnc, b,
                            part + 2 * ((long long)c.part_begin + b));
}

__global__ void multi_defect_reduce_kernel(const __grid_constant__ DefectTable tab, const double *part, double *A) {
  const int k = threadIdx.x;
  if (k >= tab.n) return;
  const DefectDesc &c = tab.c[k];
  double a1 = 0.0, a2 = 0.0;
  for (int b = 0; b < c.nblk; ++b) {
    a1 += part[2 * ((long long)c.part_begin + b)];
    a2 += part[2 * ((long long)c.part_begin + b) + 1];
  }
  A[2 * c.rep] = a1;
  A[2 * c.rep + 1] = a2;
}

__global__ void defect_sums_reduce_kernel(const double *part, int nblk, double *out) {
  if (threadIdx.x != 0) return;
  double a1 = 0.0, a2 = 0.0;
  for (int b = 0; b < nblk; ++b) {
    a1 += part[2 * b];
    a2 += part[2 * b + 1];
  }
  out[0] = a1;
  out[1] = a2;
}

int defect_sums_blocks(const Geom &g) { return (int)((g.V / g.L[0] + 255) / 256); }

cudaError_t launch_defect_sums(int nc, int dtype, const void *links, const Geom &g, const Defect &df, double beta,
                               double *d_part, double *d_out, cudaStream_t st) {
  const int nblk = defect_sums_blocks(g);
  const double bnc = beta / (double)nc;
#define KLFT_DS(NCV, NDV, TV)                                                                                   \
  defect_sums_kernel<NCV, NDV, TV><<<nblk, 256, 0, st>>>(Links<NCV, TV>{(cx<TV> *)links, g.V}, g, df, bnc, d_part)
#define KLFT_DS_ND(NCV, TV)          \
  do {                               \
    if (g.nd == 2) KLFT_DS(NCV, 2, TV); \
    else if (g.nd == 3) KLFT_DS(NCV, 3, TV); \
    else KLFT_DS(NCV, 4, TV);        \
  } while (0)
  if (dtype == 0) {
    if (nc == 1) KLFT_DS_ND(1, double);
    else if (nc == 2) KLFT_DS_ND(2, double);
    else KLFT_DS_ND(3, double);
  } else {
    if (nc == 1) KLFT_DS_ND(1, float);
    else if (nc == 2) KLFT_DS_ND(2, float);
    else KLFT_DS_ND(3, float);
  }
#undef KLFT_DS_ND
#undef KLFT_DS
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  defect_sums_reduce_kernel<<<1, 32, 0, st>>>(d_part, nblk, d_out);
  return cudaGetLastError();
}

// Sequential swap attempts of neighbouring labels (k, k+1), k = 0..nrep-2, on the
// device (one thread): the same decision rule as the host path below.
template <int NC, typename T>
static cudaError_t launch_multi_defect_nc(int nd, const DefectTable &tab, int blocks, double bnc, double *part,
                                          double *A, cudaStream_t st) {
  if (nd == 2) multi_defect_sums_kernel<NC, 2, T><<<blocks, 256, 0, st>>>(tab, bnc, part);
  else if (nd == 3) multi_defect_sums_kernel<NC, 3, T><<<blocks, 256, 0, st>>>(tab, bnc, part);
  else multi_defect_sums_kernel<NC, 4, T><<<blocks, 256, 0, st>>>(tab, bnc, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  multi_defect_reduce_kernel<<<1, 64, 0, st>>>(tab, part, A);
  return cudaGetLastError();
}

// A_1, A_2 of replica r into A[2r], A[2r + 1] for all replicas (at most 64),
// one launch pair per (Nc, Nd, precision) group; part holds
// 2 * multi_defect_parts(reps) doubles.
cudaError_t enqueue_multi_defect_sums(const std::vector<klft_lattice *> &reps, double beta, double *part, double *A,
                                      cudaStream_t st) {
  if (reps.size() > 64) return cudaErrorInvalidValue;
  std::vector<bool> done(reps.size(), false);
  int pbeg = 0;
  DefectTable tab;
  for (size_t r0 = 0; r0 < reps.size(); ++r0) {
    if (done[r0]) continue;
    const klft_lattice *k = reps[r0];
    std::memset(&tab, 0, sizeof(tab));
    int blocks = 0;
    for (size_t r = r0; r < reps.size(); ++r) {
      const klft_lattice *l = reps[r];
      if (done[r] || l->nc != k->nc || l->g.nd != k->g.nd || l->dtype() != k->dtype()) continue;
      done[r] = true;
      DefectDesc &d = tab.c[tab.n++];
      d.links = l->links;
      d.g = l->g;
      d.df = l->defect;
      d.rep = (int)r;
      d.block_begin = blocks;
      d.nblk = defect_sums_blocks(l->g);
      d.part_begin = pbeg;
      blocks += d.nblk;
      pbeg += d.nblk;
    }
    const double bnc = beta / (double)k->nc;
    const int nd = k->g.nd;
    cudaError_t e;
    if (k->dtype() == 0) {
      if (k->nc == 1) e = launch_multi_defect_nc<1, double>(nd, tab, blocks, bnc, part, A, st);
      else if (k->nc == 2) e = launch_multi_defect_nc<2, double>(nd, tab, blocks, bnc, part, A, st);
      else e = launch_multi_defect_nc<3, double>(nd, tab, blocks, bnc, part, A, st);
    } else {
      if (k->nc == 1) e = launch_multi_defect_nc<1, float>(nd, tab, blocks, bnc, part, A, st);
      else if (k->nc == 2) e = launch_multi_defect_nc<2, float>(nd, tab, blocks, bnc, part, A, st);
      else e = launch_multi_defect_nc<3, float>(nd, tab, blocks, bnc, part, A, st);
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

long long multi_defect_parts(const std::vector<klft_lattice *> &reps) {
  long long n = 0;
  for (const klft_lattice *l : reps) n += defect_sums_blocks(l->g);
  return n;
}

__global__ void ptbc_swap_kernel(int nrep, const double *c_of_label, const double *A, int *label_of_rep,
                                 int *rep_of_label, double *c_of_rep, uint64_t seed, const uint32_t *cycle_ctr,
                                 unsigned long long *swap_acc) {
  const uint32_t cycle = *cycle_ctr;
  for (int k = 0; k + 1 < nrep; ++k) {
    const int a = rep_of_label[k], b = rep_of_label[k + 1];
    const double ck = c_of_label[k], ck1 = c_of_label[k + 1];
    double dS = 0.0;
    dS += (ck - ck1) * (A[2 * b] - A[2 * a]);
    dS += (ck * ck - ck1 * ck1) * (A[2 * b + 1] - A[2 * a + 1]);
    bool acc = dS < 0.0;
    if (!acc) {
      Stream st(seed, 0, (uint32_t)k, cycle, KIND_SWAP, 0u);
      acc = st.next() < exp(-dS);
    }
    if (acc) {
      rep_of_label[k] = b;
      rep_of_label[k + 1] = a;
      label_of_rep[a] = k + 1;
      label_of_rep[b] = k;
      c_of_rep[a] = ck1;
      c_of_rep[b] = ck;
      if (swap_acc) swap_acc[k] += 1ull;
    }
  }
}

}  // namespace klft

using namespace klft;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

extern "C" {

klft_status klft_lattice_set_defect(klft_lattice *lat, int len, const int *pos, double c) {
  if (!lat) return fail(KLFT_EINVAL, "klft_lattice_set_defect: null handle");
  if (len < 0) return fail(KLFT_EINVAL, "klft_lattice_set_defect: negative length");
  if (len > 0 && !pos) return fail(KLFT_EINVAL, "klft_lattice_set_defect: null position");
  if (!(c == c)) return fail(KLFT_EINVAL, "klft_lattice_set_defect: NaN coefficient");
  std::lock_guard<std::mutex> guard(lat->mtx);
  Defect d{0, 1, {0, 0, 0}, 1.0, nullptr};
  if (len > 0) {
    d.active = 1;
    d.len = len;
    for (int k = 0; k < 3; ++k) d.pos[k] = (k + 1 < lat->g.nd) ? ((pos[k] % lat->g.L[k + 1]) + lat->g.L[k + 1]) % lat->g.L[k + 1] : 0;
    d.c = c;
  }
  lat->defect = d;
  return KLFT_OK;
}

klft_status klft_ptbc_defect_sums(klft_lattice *lat, double beta, double *out2) {
  if (!lat || !out2) return fail(KLFT_EINVAL, "klft_ptbc_defect_sums: null pointer");
  std::lock_guard<std::mutex> guard(lat->mtx);
  if (!lat->defect.active) {
    out2[0] = out2[1] = 0.0;
    return KLFT_OK;
  }
  const int nblk = defect_sums_blocks(lat->g);
  CK(lat->s_part.ensure((size_t)2 * nblk * sizeof(double)));
  CK(lat->s_out.ensure(KLFT_RESULT_SLOTS * sizeof(double)));
  CK(launch_defect_sums(lat->nc, lat->dtype(), lat->links, lat->g, lat->defect, beta, (double *)lat->s_part.ptr,
                        (double *)lat->s_out.ptr, lat->stream));
  CK(cudaMemcpyAsync(out2, lat->s_out.ptr, 2 * sizeof(double), cudaMemcpyDeviceToHost, lat->stream));
  CK(cudaStreamSynchronize(lat->stream));
  return KLFT_OK;
}

klft_status klft_ptbc_swap_sums(const double *A, int nrep, const double *c_of_label, int *label_of_rep,
                                uint64_t seed, uint32_t cycle, int *accepted) {
  if (!A || !c_of_label || !label_of_rep || nrep < 1) return fail(KLFT_EINVAL, "klft_ptbc_swap_sums: bad arguments");
  std::vector<int> seen(nrep, 0), rep_of_label(nrep);
  for (int r = 0; r < nrep; ++r) {
    const int l = label_of_rep[r];
    if (l < 0 || l >= nrep || seen[l]) return fail(KLFT_EINVAL, "klft_ptbc_swap_sums: labels are not a permutation");
    seen[l] = 1;
    rep_of_label[l] = r;
  }
  for (int k = 0; k + 1 < nrep; ++k) {
    const int a = rep_of_label[k], b = rep_of_label[k + 1];
    const double ck = c_of_label[k], ck1 = c_of_label[k + 1];
    double dS = 0.0;
    dS += (ck - ck1) * (A[2 * b] - A[2 * a]);
    dS += (ck * ck - ck1 * ck1) * (A[2 * b + 1] - A[2 * a + 1]);
    bool acc = dS < 0.0;
    if (!acc) {
      Stream st(seed, 0, (uint32_t)k, cycle, KIND_SWAP, 0u);
      acc = st.next() < std::exp(-dS);
    }
    if (accepted) accepted[k] = acc ? 1 : 0;
    if (acc) {
      rep_of_label[k] = b;
      rep_of_label[k + 1] = a;
      label_of_rep[a] = k + 1;
      label_of_rep[b] = k;
    }
  }
  return KLFT_OK;
}

klft_status klft_lattice_set_defect_c(klft_lattice *lat, double c) {
  if (!lat) return fail(KLFT_EINVAL, "klft_lattice_set_defect_c: null handle");
  if (!(c == c)) return fail(KLFT_EINVAL, "klft_lattice_set_defect_c: NaN coefficient");
  std::lock_guard<std::mutex> guard(lat->mtx);
  if (!lat->defect.active) return fail(KLFT_EINVAL, "klft_lattice_set_defect_c: the lattice has no defect");
  lat->defect.c = c;
  return KLFT_OK;
}

klft_status klft_ptbc_swap(klft_lattice *const *reps, int nrep, const double *c_of_label, int *label_of_rep,
                           double beta, uint64_t seed, uint32_t cycle, int *accepted) {
  if (!reps || !c_of_label || !label_of_rep || nrep < 1) return fail(KLFT_EINVAL, "klft_ptbc_swap: bad arguments");
  std::vector<int> seen(nrep, 0);
  for (int r = 0; r < nrep; ++r) {
    if (!reps[r]) return fail(KLFT_EINVAL, "klft_ptbc_swap: null replica %d", r);
    const int l = label_of_rep[r];
    if (l < 0 || l >= nrep || seen[l]) return fail(KLFT_EINVAL, "klft_ptbc_swap: labels are not a permutation");
    seen[l] = 1;
  }
  std::vector<double> A(2 * (size_t)nrep);
  for (int r = 0; r < nrep; ++r) {
    klft_status s = klft_ptbc_defect_sums(reps[r], beta, &A[2 * r]);
    if (s != KLFT_OK) return s;
  }
  klft_status s = klft_ptbc_swap_sums(A.data(), nrep, c_of_label, label_of_rep, seed, cycle, accepted);
  if (s != KLFT_OK) return s;
  // every replica's defect carries its (new) label's coefficient
  for (int r = 0; r < nrep; ++r) {
    std::lock_guard<std::mutex> guard(reps[r]->mtx);
    reps[r]->defect.c = c_of_label[label_of_rep[r]];
  }
  return KLFT_OK;
}

}  // extern "C"
