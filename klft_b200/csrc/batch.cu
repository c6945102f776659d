// batch.cu -- many independent chains and PTBC replicas, of uneven groups and
// extents, advanced together; one cycle (a sweep of every chain, replica swap
// attempts, plaquette of every chain) is captured once as a CUDA graph and
// replayed.
//
// Chains are grouped by kernel variant (Nc, Nd, precision, proposal, defect).
// A group's chain table travels by value in the kernel parameters (up to
// BATCH_MAX chains, read from the constant bank); its CTAs are laid out chain
// after chain, and a CTA finds its chain by a binary search on the table's
// block offsets.  Passes are the unit of ordering: for each pass val (a parity
// class of sites for the reference proposals, a link pass (mu, parity) for the
// SU(3) exp(i eps H) proposal) one launch per group updates that pass of every
// chain in the group, so every chain is swept in the order it is swept alone.
// Per-cycle results (accepted
// hits, plaquette sums, replica labels) land in device slots selected by a
// device counter, so the captured graph is replayed unchanged.  Replica swaps
// run on the device (ptbc.cu) and write each replica's defect coefficient,
// which the sweep kernels read through Defect::dyn_c.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/klft_b200.h"
#include "capi_internal.h"
#include "kernels.cuh"
#include "metropolis_site.cuh"
#include "observables.cuh"
#include "tuner.h"

namespace klft {

constexpr int BATCH_MAX = 64;

struct ChainDesc {
  void *links;
  uint32_t *ctr;  // the chain's counters ([0] = sweep)
  Geom g;
  MetroArgs a;
  Defect df;
  int index;        // chain id in the batch
  int block_begin;  // first CTA of this chain in the launch
};

struct ChainTable {
  int n;
  int nchains_total;
  int block;  // threads per CTA of the launch (<= 128)
  ChainDesc c[BATCH_MAX];
};

KLFT_D int find_chain(const ChainTable &tab) {
  int lo = 0, hi = tab.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tab.c[mid].block_begin <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// MU >= 0 (exp groups): the link pass's direction at compile time (val >> 1 == MU)
template <int NC, int ND, typename T, bool EXP, bool DF, int MU = -1>
__global__ void __launch_bounds__(128, MinBlocks<T>::v)
    multi_pass_kernel(const __grid_constant__ ChainTable tab, int val, unsigned long long *nacc_slots,
                      const uint32_t *__restrict__ slot) {
  const int ci = find_chain(tab);
  const ChainDesc &c = tab.c[ci];
  const long long t = (long long)(blockIdx.x - c.block_begin) * blockDim.x + threadIdx.x;
  int nacc = 0;
  const Links<NC, T> U{(cx<T> *)c.links, c.g.V};
  if constexpr (EXP && NC == 3) {
    bool ok = false;
    const Site x = link_pass_site(c.g, t, val & 1, ND, ok);
    if (ok && t < link_pass_threads(c.g, ND))
      nacc = link_update_exp<ND, T, DF, MU>(U, c.g, x, MU, c.a, *c.ctr, c.df);
  } else {
    if (t < c.g.Vh) nacc = site_update_ref<NC, ND, T, DF>(U, c.g, pass_site(c.g, t, val, ND), c.a, *c.ctr, c.df);
  }
  add_accepts(nacc, nacc_slots + (size_t)(*slot) * tab.nchains_total + c.index);
}

__global__ void batch_advance_kernel(uint32_t *const *ctrs, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ctrs[i][0] += 1u;
}

// sweep counters of up to CtrList::MAX lattices, passed by value
struct CtrList {
  static constexpr int MAX = 128;
  int n;
  uint32_t *p[MAX];
};

__global__ void advance_list_kernel(const __grid_constant__ CtrList l) {
  if ((int)threadIdx.x < l.n) l.p[threadIdx.x][0] += 1u;
}

__global__ void batch_slot_kernel(uint32_t *slot, uint32_t *cycle) {
  *slot += 1u;
  *cycle += 1u;
}

__global__ void copy_labels_kernel(const int *labels, int n, int *dst, const uint32_t *slot) {
  const int i = threadIdx.x;
  if (i < n) dst[(size_t)(*slot) * n + i] = labels[i];
}

// Plaquette sums of up to BATCH_MAX lattices of one (Nc, Nd, precision) in one
// launch: chain k owns CTAs [block_begin, block_begin + nblk) and partials
// [part_begin, part_begin + nblk).  Each CTA computes exactly the partial that
// block (blockIdx.x - block_begin) of the single-lattice plaquette launch writes
// and multi_reduce_kernel sums them in the single-lattice order, so a chain's
// sum in a batch is bit-identical to its solo plaquette.
struct PlaqDesc {
  void *links;
  Geom g;
  long long part_begin;
  int index;  // column of the chain in the result slots
  int block_begin;
  int nblk;
};

struct PlaqTable {
  int n;
  PlaqDesc c[BATCH_MAX];
};

template <int NC, int ND, typename T>
__global__ void __launch_bounds__(RED_THREADS, PlaqMinBlocks<T>::v)
    multi_plaquette_kernel(const __grid_constant__ PlaqTable tab, double *__restrict__ part) {
  int lo = 0, hi = tab.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tab.c[mid].block_begin <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const PlaqDesc &c = tab.c[lo];
  const int b = (int)blockIdx.x - c.block_begin;
  const double s = block_sum<RED_THREADS>(
      plaquette_partial<NC, ND, T>(Links<NC, T>{(cx<T> *)c.links, c.g.V}, c.g, ND, b, c.nblk));
  if (threadIdx.x == 0) part[c.part_begin + b] = s;
}

// one CTA per chain of the table: plaq[(*slot) * stride + index] = sum of its partials
__global__ void multi_reduce_kernel(const __grid_constant__ PlaqTable tab, const double *__restrict__ part,
                                    double *plaq, const uint32_t *slot, int stride) {
  const PlaqDesc &c = tab.c[blockIdx.x];
  double v = 0.0;
  for (int i = threadIdx.x; i < c.nblk; i += RED_THREADS) v += part[c.part_begin + i];
  const double s = block_sum<RED_THREADS>(v);
  if (threadIdx.x == 0) plaq[(size_t)(*slot) * stride + c.index] = s;
}

template <int NC, typename T>
cudaError_t launch_multi_plaquette_nc(int nd, const PlaqTable &tab, int blocks, double *part, double *plaq,
                                      const uint32_t *slot, int stride, cudaStream_t st) {
  if (nd == 2) multi_plaquette_kernel<NC, 2, T><<<blocks, RED_THREADS, 0, st>>>(tab, part);
  else if (nd == 3) multi_plaquette_kernel<NC, 3, T><<<blocks, RED_THREADS, 0, st>>>(tab, part);
  else multi_plaquette_kernel<NC, 4, T><<<blocks, RED_THREADS, 0, st>>>(tab, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  multi_reduce_kernel<<<tab.n, RED_THREADS, 0, st>>>(tab, part, plaq, slot, stride);
  return cudaGetLastError();
}

// Plaquette sums of all lattices into plaq[(*slot) * stride + index_i], one
// multi-chain launch pair per (Nc, Nd, precision) group of up to BATCH_MAX;
// part holds sum_i plaquette_blocks(g_i) doubles.
cudaError_t enqueue_multi_plaquette(const std::vector<klft_lattice *> &lats, const std::vector<int> &index,
                                    double *part, double *plaq, const uint32_t *slot, int stride, cudaStream_t st,
                                    int *nlaunch) {
  struct Key {
    int nc, nd, dtype;
  };
  std::vector<Key> keys;
  std::vector<std::vector<int>> members;
  for (size_t i = 0; i < lats.size(); ++i) {
    const Key k{lats[i]->nc, lats[i]->g.nd, lats[i]->dtype()};
    size_t gi = 0;
    while (gi < keys.size() && !(keys[gi].nc == k.nc && keys[gi].nd == k.nd && keys[gi].dtype == k.dtype)) ++gi;
    if (gi == keys.size()) {
      keys.push_back(k);
      members.emplace_back();
    }
    members[gi].push_back((int)i);
  }
  long long pbeg = 0;
  std::unique_ptr<PlaqTable> tab(new PlaqTable());
  for (size_t gi = 0; gi < keys.size(); ++gi)
    for (size_t m0 = 0; m0 < members[gi].size(); m0 += BATCH_MAX) {
      std::memset(tab.get(), 0, sizeof(PlaqTable));
      int blocks = 0;
      for (size_t m = m0; m < members[gi].size() && m < m0 + BATCH_MAX; ++m) {
        const int i = members[gi][m];
        PlaqDesc &d = tab->c[tab->n++];
        d.links = lats[i]->links;
        d.g = lats[i]->g;
        d.part_begin = pbeg;
        d.index = index[i];
        d.block_begin = blocks;
        d.nblk = plaquette_blocks(d.g);
        blocks += d.nblk;
        pbeg += d.nblk;
      }
      const Key &k = keys[gi];
      cudaError_t e;
      if (k.dtype == 0) {
        if (k.nc == 1) e = launch_multi_plaquette_nc<1, double>(k.nd, *tab, blocks, part, plaq, slot, stride, st);
        else if (k.nc == 2) e = launch_multi_plaquette_nc<2, double>(k.nd, *tab, blocks, part, plaq, slot, stride, st);
        else e = launch_multi_plaquette_nc<3, double>(k.nd, *tab, blocks, part, plaq, slot, stride, st);
      } else {
        if (k.nc == 1) e = launch_multi_plaquette_nc<1, float>(k.nd, *tab, blocks, part, plaq, slot, stride, st);
        else if (k.nc == 2) e = launch_multi_plaquette_nc<2, float>(k.nd, *tab, blocks, part, plaq, slot, stride, st);
        else e = launch_multi_plaquette_nc<3, float>(k.nd, *tab, blocks, part, plaq, slot, stride, st);
      }
      if (e != cudaSuccess) return e;
      if (nlaunch) *nlaunch += 2;
    }
  return cudaSuccess;
}

long long multi_plaquette_parts(const std::vector<klft_lattice *> &lats) {
  long long n = 0;
  for (klft_lattice *l : lats) n += plaquette_blocks(l->g);
  return n;
}

// declared in ptbc.cu
cudaError_t enqueue_multi_defect_sums(const std::vector<klft_lattice *> &reps, double beta, double *part, double *A,
                                      cudaStream_t st);
long long multi_defect_parts(const std::vector<klft_lattice *> &reps);
__global__ void ptbc_swap_kernel(int nrep, const double *c_of_label, const double *A, int *label_of_rep,
                                 int *rep_of_label, double *c_of_rep, uint64_t seed, const uint32_t *cycle_ctr,
                                 unsigned long long *swap_acc);

}  // namespace klft

using namespace klft;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

struct klft_batch {
  struct Chain {
    klft_lattice *lat;
    double beta, delta, eps;
    int nhits, proposal;
  };
  static constexpr int NSIDE = 3;
  int device = 0;
  cudaStream_t stream = nullptr;
  // side streams for the sweep launches of the second and later chain groups
  cudaStream_t side[NSIDE] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[NSIDE] = {};
  std::vector<Chain> chains;
  // PTBC
  std::vector<int> reps;  // chain ids of the replicas, replica r = reps[r]
  std::vector<double> c_of_label;
  double ptbc_beta = 0.0;
  uint64_t swap_seed = 0;
  // device state
  uint32_t *d_slot = nullptr;   // [0] result slot, [1] cycle counter (swap stream step)
  uint32_t **d_ctrs = nullptr;  // per-chain counter pointers
  double *d_c_of_label = nullptr, *d_c_of_rep = nullptr, *d_A = nullptr, *d_part = nullptr;
  int *d_label_of_rep = nullptr, *d_rep_of_label = nullptr;
  unsigned long long *d_swap_acc = nullptr;
  klft::Scratch s_nacc, s_plaq, s_labels, s_ppart, s_tune;
  int sweep_block = 128;  // threads per CTA of the sweep launches (tuned under KLFT_TUNING)
  int cap = 0;  // result slots
  bool dirty = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_measure = -1;
  std::mutex mtx;

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
};

namespace {

struct GroupKey {
  int nc, nd, dtype, exp, df;
  bool operator==(const GroupKey &o) const {
    return nc == o.nc && nd == o.nd && dtype == o.dtype && exp == o.exp && df == o.df;
  }
};

template <int NC, int ND, typename T, bool EXP, bool DF>
cudaError_t launch_group_t(const ChainTable &tab, int blocks, int val, unsigned long long *nacc, const uint32_t *slot,
                           cudaStream_t st) {
  if constexpr (EXP && NC == 3) {
    // one kernel instance per link direction (compiled staple site steps)
    switch (val >> 1) {
      case 0: multi_pass_kernel<NC, ND, T, EXP, DF, 0><<<blocks, tab.block, 0, st>>>(tab, val, nacc, slot); break;
      case 1: multi_pass_kernel<NC, ND, T, EXP, DF, 1><<<blocks, tab.block, 0, st>>>(tab, val, nacc, slot); break;
      case 2:
        if constexpr (ND > 2)
          multi_pass_kernel<NC, ND, T, EXP, DF, (ND > 2 ? 2 : 0)><<<blocks, tab.block, 0, st>>>(tab, val, nacc, slot);
        break;
      default:
        if constexpr (ND > 3)
          multi_pass_kernel<NC, ND, T, EXP, DF, (ND > 3 ? 3 : 0)><<<blocks, tab.block, 0, st>>>(tab, val, nacc, slot);
        break;
    }
  } else {
    multi_pass_kernel<NC, ND, T, EXP, DF><<<blocks, tab.block, 0, st>>>(tab, val, nacc, slot);
  }
  return cudaGetLastError();
}

template <int NC, int ND, typename T>
cudaError_t launch_group_nd(const GroupKey &k, const ChainTable &tab, int blocks, int val, unsigned long long *nacc,
                            const uint32_t *slot, cudaStream_t st) {
  if (k.exp) {
    if (k.df) return launch_group_t<NC, ND, T, true, true>(tab, blocks, val, nacc, slot, st);
    return launch_group_t<NC, ND, T, true, false>(tab, blocks, val, nacc, slot, st);
  }
  if (k.df) return launch_group_t<NC, ND, T, false, true>(tab, blocks, val, nacc, slot, st);
  return launch_group_t<NC, ND, T, false, false>(tab, blocks, val, nacc, slot, st);
}

template <int NC, typename T>
cudaError_t launch_group_nc(const GroupKey &k, const ChainTable &tab, int blocks, int val, unsigned long long *nacc,
                            const uint32_t *slot, cudaStream_t st) {
  if (k.nd == 2) return launch_group_nd<NC, 2, T>(k, tab, blocks, val, nacc, slot, st);
  if (k.nd == 3) return launch_group_nd<NC, 3, T>(k, tab, blocks, val, nacc, slot, st);
  return launch_group_nd<NC, 4, T>(k, tab, blocks, val, nacc, slot, st);
}

cudaError_t launch_group(const GroupKey &k, const ChainTable &tab, int blocks, int val, unsigned long long *nacc,
                         const uint32_t *slot, cudaStream_t st) {
  if (k.dtype == 0) {
    if (k.nc == 1) return launch_group_nc<1, double>(k, tab, blocks, val, nacc, slot, st);
    if (k.nc == 2) return launch_group_nc<2, double>(k, tab, blocks, val, nacc, slot, st);
    return launch_group_nc<3, double>(k, tab, blocks, val, nacc, slot, st);
  }
  if (k.nc == 1) return launch_group_nc<1, float>(k, tab, blocks, val, nacc, slot, st);
  if (k.nc == 2) return launch_group_nc<2, float>(k, tab, blocks, val, nacc, slot, st);
  return launch_group_nc<3, float>(k, tab, blocks, val, nacc, slot, st);
}

struct Group {
  GroupKey key;
  std::vector<std::unique_ptr<ChainTable>> tables;
  std::vector<int> blocks;
};

}  // namespace

namespace klft {

// One sweep of every item, interleaved by pass, in multi-chain launches
// on stream st.  Accepted hits of item i go to nacc[(*slot) * stride + index],
// index = items[i].acc_index (i when negative), stride = acc_stride (n when 0);
// the caller advances the items' sweep counters afterwards.
klft_status enqueue_multi_sweep(const std::vector<SweepItem> &items, unsigned long long *nacc, const uint32_t *slot,
                                cudaStream_t st, int acc_stride, int *nlaunch, const StreamFork *fork, int block) {
  if (block != 32 && block != 64 && block != 128) return fail(KLFT_EINVAL, "enqueue_multi_sweep: block %d", block);
  const int n = (int)items.size();
  const int stride = acc_stride > 0 ? acc_stride : n;
  std::vector<Group> groups;
  for (int i = 0; i < n; ++i) {
    const SweepItem &it = items[i];
    klft_lattice *lat = it.lat;
    GroupKey key{lat->nc, lat->g.nd, lat->dtype(), (lat->nc == 3 && it.a.proposal == KLFT_PROPOSAL_EXP) ? 1 : 0,
                 it.df.active ? 1 : 0};
    Group *grp = nullptr;
    for (auto &gg : groups)
      if (gg.key == key) grp = &gg;
    if (!grp) {
      groups.push_back(Group{key, {}, {}});
      grp = &groups.back();
    }
    if (grp->tables.empty() || grp->tables.back()->n == BATCH_MAX) {
      grp->tables.emplace_back(new ChainTable());
      std::memset(grp->tables.back().get(), 0, sizeof(ChainTable));
      grp->tables.back()->nchains_total = stride;
      grp->tables.back()->block = block;
      grp->blocks.push_back(0);
    }
    ChainTable &tab = *grp->tables.back();
    ChainDesc &d = tab.c[tab.n++];
    d.links = lat->links;
    d.ctr = lat->d_counters;
    d.g = lat->g;
    d.a = it.a;
    if (key.dtype == 0 && key.exp && !(d.a.bm = bm_table()))
      return fail(KLFT_ECUDA, "enqueue_multi_sweep: Box-Muller table unavailable");
    d.df = it.df;
    d.index = it.acc_index >= 0 ? it.acc_index : i;
    d.block_begin = grp->blocks.back();
    // exp groups: V/2 links per link pass; reference groups: Vh sites per class
    const long long nthr = key.exp ? link_pass_threads(lat->g, lat->g.nd) : lat->g.Vh;
    grp->blocks.back() += (int)((nthr + block - 1) / block);
  }
  int maxpass = 0;
  for (auto &gg : groups) {
    const int np = gg.key.exp ? 2 * gg.key.nd : 1 << gg.key.nd;
    maxpass = np > maxpass ? np : maxpass;
  }
  const int ng = (int)groups.size();
  const int nside = fork && ng > 1 ? std::min(fork->nside, ng - 1) : 0;
  if (nside > 0) {
    CK(cudaEventRecord(fork->fork, st));
    for (int i = 0; i < nside; ++i) CK(cudaStreamWaitEvent(fork->side[i], fork->fork, 0));
  }
  // the side streams are joined back even when a launch fails
  cudaError_t err = cudaSuccess;
  for (int val = 0; val < maxpass && err == cudaSuccess; ++val)
    for (int gi = 0; gi < ng && err == cudaSuccess; ++gi) {
      const Group &gg = groups[gi];
      if (val >= (gg.key.exp ? 2 * gg.key.nd : 1 << gg.key.nd)) continue;
      const cudaStream_t gs = gi == 0 || nside == 0 ? st : fork->side[(gi - 1) % nside];
      for (size_t t = 0; t < gg.tables.size() && err == cudaSuccess; ++t) {
        err = launch_group(gg.key, *gg.tables[t], gg.blocks[t], val, nacc, slot, gs);
        if (nlaunch) ++*nlaunch;
      }
    }
  for (int i = 0; i < nside; ++i) {
    const cudaError_t e1 = cudaEventRecord(fork->join[i], fork->side[i]);
    const cudaError_t e2 = cudaStreamWaitEvent(st, fork->join[i], 0);
    if (err == cudaSuccess) err = e1 != cudaSuccess ? e1 : e2;
  }
  if (err != cudaSuccess) return cuda_fail(err, "enqueue_multi_sweep");
  return KLFT_OK;
}

cudaError_t launch_advance_many(uint32_t *const *d_ctrs, int n, cudaStream_t st) {
  batch_advance_kernel<<<(n + 127) / 128, 128, 0, st>>>(d_ctrs, n);
  return cudaGetLastError();
}

cudaError_t launch_advance_list(const std::vector<uint32_t *> &ctrs, cudaStream_t st, int *nlaunch) {
  for (size_t b = 0; b < ctrs.size(); b += CtrList::MAX) {
    CtrList l;
    l.n = (int)std::min(ctrs.size() - b, (size_t)CtrList::MAX);
    for (int i = 0; i < l.n; ++i) l.p[i] = ctrs[b + i];
    advance_list_kernel<<<1, CtrList::MAX, 0, st>>>(l);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (nlaunch) ++*nlaunch;
  }
  return cudaSuccess;
}

}  // namespace klft

namespace {

// The sweep items of every chain (replicas read their coefficient from the device).
std::vector<SweepItem> sweep_items(const klft_batch *b) {
  const int n = (int)b->chains.size();
  std::vector<SweepItem> items;
  for (int i = 0; i < n; ++i) {
    const auto &ch = b->chains[i];
    klft_lattice *lat = ch.lat;
    SweepItem it{lat, MetroArgs{ch.beta, ch.delta, ch.eps, ch.nhits, ch.proposal, lat->seed, lat->chain},
                 lat->defect, -1};
    for (size_t r = 0; r < b->reps.size(); ++r)
      if (b->reps[r] == i) it.df.dyn_c = b->d_c_of_rep + r;
    items.push_back(it);
  }
  return items;
}

// Enqueue one cycle on b->stream (recorded into the graph by the caller).
klft_status enqueue_cycle(klft_batch *b, int measure) {
  const int n = (int)b->chains.size();
  const std::vector<SweepItem> items = sweep_items(b);
  const StreamFork fork{b->ev_fork, b->side, b->ev_join, klft_batch::NSIDE};
  klft_status st = enqueue_multi_sweep(items, (unsigned long long *)b->s_nacc.ptr, b->d_slot, b->stream, 0, nullptr,
                                       &fork, b->sweep_block);
  if (st != KLFT_OK) return st;
  CK(launch_advance_many(b->d_ctrs, n, b->stream));
  if (!b->reps.empty()) {
    const int nrep = (int)b->reps.size();
    std::vector<klft_lattice *> reps;
    for (int r = 0; r < nrep; ++r) reps.push_back(b->chains[b->reps[r]].lat);
    CK(enqueue_multi_defect_sums(reps, b->ptbc_beta, b->d_part, b->d_A, b->stream));
    ptbc_swap_kernel<<<1, 1, 0, b->stream>>>(nrep, b->d_c_of_label, b->d_A, b->d_label_of_rep, b->d_rep_of_label,
                                             b->d_c_of_rep, b->swap_seed, b->d_slot + 1, b->d_swap_acc);
    CK(cudaGetLastError());
    copy_labels_kernel<<<1, 64, 0, b->stream>>>(b->d_label_of_rep, nrep, (int *)b->s_labels.ptr, b->d_slot);
    CK(cudaGetLastError());
  }
  if (measure) {
    std::vector<klft_lattice *> lats;
    std::vector<int> index;
    for (int i = 0; i < n; ++i) {
      lats.push_back(b->chains[i].lat);
      index.push_back(i);
    }
    CK(enqueue_multi_plaquette(lats, index, (double *)b->s_ppart.ptr, (double *)b->s_plaq.ptr, b->d_slot, n,
                               b->stream, nullptr));
  }
  batch_slot_kernel<<<1, 1, 0, b->stream>>>(b->d_slot, b->d_slot + 1);
  CK(cudaGetLastError());
  return KLFT_OK;
}

// Under KLFT_TUNING: the CTA size of the batch's sweep launches (32, 64 or 128
// threads), tuned once per batch composition (key: chain count and a hash of
// every chain's group, extents, precision, proposal and defect) and cached like
// the single-lattice sweep.  Candidates are timed on the chains' own links,
// which are backed up first and restored afterwards; counters do not move, so
// no chain is perturbed.  Results never depend on the block size.
klft_status tune_sweep_block(klft_batch *b) {
  b->sweep_block = 128;
  if (!tuner_enabled()) return KLFT_OK;
  const int n = (int)b->chains.size();
  uint64_t h = 1469598103934665603ull;
  auto mix = [&h](long long v) {
    h ^= (uint64_t)v;
    h *= 1099511628211ull;
  };
  long long sites = 0;
  size_t total = 0;
  for (const auto &ch : b->chains) {
    const klft_lattice *l = ch.lat;
    mix(l->nc);
    mix(l->g.nd);
    for (int d = 0; d < 4; ++d) mix(l->g.L[d]);
    mix(l->dtype());
    mix(ch.proposal);
    mix(l->defect.active);
    sites += l->g.Vh;
    total += (l->link_bytes + 255) & ~(size_t)255;
  }
  char hex[17];
  snprintf(hex, sizeof hex, "%016llx", (unsigned long long)h);
  const std::string id = "sweep_Metropolis_batch_" + std::to_string(n) + "_chains_" + hex;
  const int end[1] = {(int)std::min<long long>(sites, 2147483647LL)};
  const std::string key = tune_key(id, 1, end);
  const std::vector<SweepItem> items = sweep_items(b);
  auto time_fn = [&](int block) -> float {
    if (b->s_tune.ensure(total) != cudaSuccess) return -1.f;
    char *bak = (char *)b->s_tune.ptr;
    size_t off = 0;
    for (const auto &ch : b->chains) {
      if (cudaMemcpyAsync(bak + off, ch.lat->links, ch.lat->link_bytes, cudaMemcpyDeviceToDevice, b->stream) !=
          cudaSuccess)
        return -1.f;
      off += (ch.lat->link_bytes + 255) & ~(size_t)255;
    }
    if (cudaMemsetAsync(b->d_slot, 0, sizeof(uint32_t), b->stream) != cudaSuccess) return -1.f;
    const float ms = time_launches(b->stream, 3, [&] {
      return enqueue_multi_sweep(items, (unsigned long long *)b->s_nacc.ptr, b->d_slot, b->stream, n, nullptr,
                                 nullptr, block) == KLFT_OK
                 ? cudaSuccess
                 : cudaErrorLaunchFailure;
    });
    off = 0;
    for (const auto &ch : b->chains) {
      if (cudaMemcpyAsync(ch.lat->links, bak + off, ch.lat->link_bytes, cudaMemcpyDeviceToDevice, b->stream) !=
          cudaSuccess)
        return -1.f;
      off += (ch.lat->link_bytes + 255) & ~(size_t)255;
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return -1.f;
    return ms;
  };
  b->sweep_block = tuned_param(key, 1, {32, 64, 128}, 128, time_fn, true);
  b->s_tune.release();
  CK(cudaGetLastError());
  return KLFT_OK;
}

klft_status prepare(klft_batch *b, int ncycles) {
  const int n = (int)b->chains.size();
  if (ncycles > b->cap) {
    b->cap = ncycles;
    b->dirty = true;
  }
  CK(b->s_nacc.ensure((size_t)b->cap * n * sizeof(unsigned long long)));
  CK(b->s_plaq.ensure((size_t)b->cap * n * sizeof(double)));
  CK(b->s_labels.ensure((size_t)b->cap * (b->reps.empty() ? 1 : b->reps.size()) * sizeof(int)));
  std::vector<klft_lattice *> lats;
  for (auto &ch : b->chains) lats.push_back(ch.lat);
  CK(b->s_ppart.ensure((size_t)(multi_plaquette_parts(lats) + 1) * sizeof(double)));
  if (!b->d_ctrs) {
    CK(cudaMalloc(&b->d_ctrs, BATCH_MAX * 64 * sizeof(uint32_t *)));
  }
  std::vector<uint32_t *> ctrs;
  for (auto &ch : b->chains) ctrs.push_back(ch.lat->d_counters);
  CK(cudaMemcpyAsync(b->d_ctrs, ctrs.data(), ctrs.size() * sizeof(uint32_t *), cudaMemcpyHostToDevice, b->stream));
  return KLFT_OK;
}

}  // namespace

extern "C" {

klft_status klft_batch_create(klft_batch **out) {
  if (!out) return fail(KLFT_EINVAL, "klft_batch_create: null pointer");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(KLFT_ECUDA, "klft_batch_create: no CUDA device available");
  klft_batch *b = new klft_batch();
  cudaGetDevice(&b->device);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  for (int i = 0; i < klft_batch::NSIDE && e == cudaSuccess; ++i) {
    e = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_slot, 4 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_slot, 0, 4 * sizeof(uint32_t), b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) {
    klft_status s = cuda_fail(e, "klft_batch_create");
    klft_batch_destroy(b);
    return s;
  }
  *out = b;
  return KLFT_OK;
}

klft_status klft_batch_destroy(klft_batch *b) {
  if (!b) return KLFT_OK;
  {
    std::lock_guard<std::mutex> g(b->mtx);
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->drop_graph();
    for (klft::Scratch *s : {&b->s_nacc, &b->s_plaq, &b->s_labels, &b->s_ppart, &b->s_tune}) s->release();
    for (void *p : {(void *)b->d_slot, (void *)b->d_ctrs, (void *)b->d_c_of_label, (void *)b->d_c_of_rep,
                    (void *)b->d_A, (void *)b->d_part, (void *)b->d_label_of_rep, (void *)b->d_rep_of_label,
                    (void *)b->d_swap_acc})
      if (p) cudaFree(p);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (int i = 0; i < klft_batch::NSIDE; ++i) {
      if (b->side[i]) cudaStreamDestroy(b->side[i]);
      if (b->ev_join[i]) cudaEventDestroy(b->ev_join[i]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  }
  delete b;
  return KLFT_OK;
}

klft_status klft_batch_add_chain(klft_batch *b, klft_lattice *lat, double beta, double delta, int nhits, int proposal,
                                 double eps, int *chain_id) {
  if (!b || !lat) return fail(KLFT_EINVAL, "klft_batch_add_chain: null handle");
  if (nhits < 0) return fail(KLFT_EINVAL, "klft_batch_add_chain: negative nHits");
  if (proposal != KLFT_PROPOSAL_REFERENCE && proposal != KLFT_PROPOSAL_EXP)
    return fail(KLFT_EINVAL, "klft_batch_add_chain: unknown proposal %d", proposal);
  if (lat->nc == 3 && proposal == KLFT_PROPOSAL_REFERENCE && !(delta > 0.0))
    return fail(KLFT_EINVAL, "klft_batch_add_chain: the reference SU(3) proposal needs delta > 0");
  if (lat->device != b->device) return fail(KLFT_EINVAL, "klft_batch_add_chain: lattice on another device");
  std::lock_guard<std::mutex> g(b->mtx);
  if (b->chains.size() >= (size_t)BATCH_MAX * 64) return fail(KLFT_EINVAL, "klft_batch_add_chain: too many chains");
  for (auto &ch : b->chains)
    if (ch.lat == lat) return fail(KLFT_EINVAL, "klft_batch_add_chain: lattice already in the batch");
  b->chains.push_back({lat, beta, delta, eps, nhits, proposal});
  if (chain_id) *chain_id = (int)b->chains.size() - 1;
  b->dirty = true;
  return KLFT_OK;
}

klft_status klft_batch_set_ptbc(klft_batch *b, const int *chain_ids, int nrep, const double *c_of_label, double beta,
                                uint64_t swap_seed) {
  if (!b || !chain_ids || !c_of_label || nrep < 1 || nrep > 64)
    return fail(KLFT_EINVAL, "klft_batch_set_ptbc: bad arguments (1 <= nrep <= 64)");
  std::lock_guard<std::mutex> g(b->mtx);
  for (int r = 0; r < nrep; ++r) {
    if (chain_ids[r] < 0 || chain_ids[r] >= (int)b->chains.size())
      return fail(KLFT_EINVAL, "klft_batch_set_ptbc: unknown chain %d", chain_ids[r]);
    if (!b->chains[chain_ids[r]].lat->defect.active)
      return fail(KLFT_EINVAL, "klft_batch_set_ptbc: chain %d has no defect (klft_lattice_set_defect)", chain_ids[r]);
  }
  b->reps.assign(chain_ids, chain_ids + nrep);
  b->c_of_label.assign(c_of_label, c_of_label + nrep);
  b->ptbc_beta = beta;
  b->swap_seed = swap_seed;
  for (void **p : {(void **)&b->d_c_of_label, (void **)&b->d_c_of_rep, (void **)&b->d_A, (void **)&b->d_part,
                   (void **)&b->d_label_of_rep, (void **)&b->d_rep_of_label, (void **)&b->d_swap_acc})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
  std::vector<klft_lattice *> replats;
  for (int r = 0; r < nrep; ++r) replats.push_back(b->chains[chain_ids[r]].lat);
  CK(cudaMalloc(&b->d_c_of_label, nrep * sizeof(double)));
  CK(cudaMalloc(&b->d_c_of_rep, nrep * sizeof(double)));
  CK(cudaMalloc(&b->d_A, 2 * nrep * sizeof(double)));
  CK(cudaMalloc(&b->d_part, 2 * (size_t)multi_defect_parts(replats) * sizeof(double)));
  CK(cudaMalloc(&b->d_label_of_rep, nrep * sizeof(int)));
  CK(cudaMalloc(&b->d_rep_of_label, nrep * sizeof(int)));
  CK(cudaMalloc(&b->d_swap_acc, nrep * sizeof(unsigned long long)));
  std::vector<int> lab(nrep);
  for (int r = 0; r < nrep; ++r) lab[r] = r;
  CK(cudaMemcpyAsync(b->d_c_of_label, c_of_label, nrep * sizeof(double), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->d_c_of_rep, c_of_label, nrep * sizeof(double), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->d_label_of_rep, lab.data(), nrep * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->d_rep_of_label, lab.data(), nrep * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemsetAsync(b->d_swap_acc, 0, nrep * sizeof(unsigned long long), b->stream));
  CK(cudaStreamSynchronize(b->stream));
  b->dirty = true;
  return KLFT_OK;
}

klft_status klft_batch_run(klft_batch *b, int ncycles, int measure_plaquette, int use_graph, double *acc_out,
                           double *plaq_out, int *labels_out, double *device_ms) {
  if (!b) return fail(KLFT_EINVAL, "klft_batch_run: null handle");
  if (ncycles < 0) return fail(KLFT_EINVAL, "klft_batch_run: negative count");
  if (b->chains.empty()) return fail(KLFT_EINVAL, "klft_batch_run: no chains");
  if (ncycles == 0) return KLFT_OK;
  std::lock_guard<std::mutex> guard(b->mtx);
  const int n = (int)b->chains.size();
  const int nrep = (int)b->reps.size();
  // member lattices must be idle: their own streams may still hold work
  for (auto &ch : b->chains) CK(cudaStreamSynchronize(ch.lat->stream));
  klft_status s = prepare(b, ncycles);
  if (s != KLFT_OK) return s;
  if (b->dirty) {
    s = tune_sweep_block(b);
    if (s != KLFT_OK) return s;
  }
  if (b->dirty || b->graph_measure != measure_plaquette) b->drop_graph();
  CK(cudaMemsetAsync(b->d_slot, 0, sizeof(uint32_t), b->stream));
  CK(cudaMemsetAsync(b->s_nacc.ptr, 0, (size_t)ncycles * n * sizeof(unsigned long long), b->stream));
  if (use_graph && !b->exec) {
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    s = enqueue_cycle(b, measure_plaquette);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (s != KLFT_OK) {
      if (graph) cudaGraphDestroy(graph);
      return s;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    b->graph = graph;
    CK(cudaGraphInstantiate(&b->exec, graph, 0));
    b->graph_measure = measure_plaquette;
    b->dirty = false;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, b->stream));
  for (int c = 0; c < ncycles; ++c) {
    if (use_graph) {
      CK(cudaGraphLaunch(b->exec, b->stream));
    } else {
      s = enqueue_cycle(b, measure_plaquette);
      if (s != KLFT_OK) return s;
    }
  }
  CK(cudaEventRecord(e1, b->stream));
  std::vector<unsigned long long> h_nacc((size_t)ncycles * n);
  CK(cudaMemcpyAsync(h_nacc.data(), b->s_nacc.ptr, h_nacc.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     b->stream));
  if (plaq_out && measure_plaquette)
    CK(cudaMemcpyAsync(plaq_out, b->s_plaq.ptr, (size_t)ncycles * n * sizeof(double), cudaMemcpyDeviceToHost,
                       b->stream));
  if (labels_out && nrep > 0)
    CK(cudaMemcpyAsync(labels_out, b->s_labels.ptr, (size_t)ncycles * nrep * sizeof(int), cudaMemcpyDeviceToHost,
                       b->stream));
  CK(cudaStreamSynchronize(b->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (device_ms) *device_ms = ms;
  for (int i = 0; i < n; ++i) {
    klft_lattice *lat = b->chains[i].lat;
    double norm = 1.0;
    for (int d = 0; d < lat->g.nd; ++d) norm *= (double)lat->g.L[d];
    norm *= (double)lat->g.nd;
    norm *= (double)b->chains[i].nhits;
    for (int c = 0; c < ncycles; ++c) {
      if (acc_out) acc_out[(size_t)c * n + i] = b->chains[i].nhits ? (double)h_nacc[(size_t)c * n + i] / norm : 0.0;
      if (plaq_out && measure_plaquette) plaq_out[(size_t)c * n + i] = normalize_plaquette(lat, plaq_out[(size_t)c * n + i]);
    }
  }
  // the replicas' host-side defect coefficients follow the device labels
  if (nrep > 0) {
    std::vector<double> crep(nrep);
    CK(cudaMemcpy(crep.data(), b->d_c_of_rep, nrep * sizeof(double), cudaMemcpyDeviceToHost));
    for (int r = 0; r < nrep; ++r) b->chains[b->reps[r]].lat->defect.c = crep[r];
  }
  return KLFT_OK;
}

klft_status klft_batch_swap_stats(klft_batch *b, unsigned long long *accepted_per_pair) {
  if (!b || !accepted_per_pair) return fail(KLFT_EINVAL, "klft_batch_swap_stats: null pointer");
  std::lock_guard<std::mutex> guard(b->mtx);
  const int nrep = (int)b->reps.size();
  if (nrep == 0) return KLFT_OK;
  CK(cudaMemcpy(accepted_per_pair, b->d_swap_acc, (size_t)(nrep - 1 > 0 ? nrep - 1 : 0) * sizeof(unsigned long long),
                cudaMemcpyDeviceToHost));
  return KLFT_OK;
}

}  // extern "C"
