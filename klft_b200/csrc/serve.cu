// serve.cu -- continuous-batching job server over device-resident lattices.
//
// The reference runs one simulation per process (Metropolis.hpp:113-223,
// HMC.hpp:20-117); this file has no counterpart there.  It keeps many jobs'
// lattices and Philox counters resident in HBM and advances them together:
//
//   * admission: a FIFO queue; the head job is admitted when its device
//     footprint fits the budget and a running slot is free.  Its lattice is
//     created and every buffer it will touch is sized at admission, so nothing
//     allocates while GPU work of other jobs is being enqueued.
//   * Metropolis rounds: every running Metropolis job gets one sweep per round
//     step, all jobs of a step in multi-chain launches (one per parity class
//     and lattice group, enqueue_multi_sweep), then one counter-advance
//     launch.  Jobs are split into kClasses size classes by the cost of a sweep,
//     each with its own round pipeline on its own stream, so small (latency-
//     bound) lattices do not wait for the sweeps of large ones and run beside
//     them.  kRoundsInFlight rounds are queued ahead per class, so a job that
//     arrives while a round runs joins its class's next round.
//   * HMC jobs run trajectory by trajectory on their lattice's own stream, at
//     most kTrajAhead trajectories ahead, overlapping the rounds.
//   * a finished job is measured on its own stream (after the round holding its
//     last sweep), the results land in its pinned result slots, and the worker
//     posts them once the job's event has completed.
//
// Every kernel a job runs is the one that would run for it alone, on its own
// lattice, with counter-based random numbers keyed on (seed, chain, sweep or
// trajectory, site), so its result does not depend on what else is running.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/klft_b200.h"
#include "capi_internal.h"
#include "kernels.cuh"

using namespace klft;

namespace {

constexpr int kSweepsPerRound = 4;  // round steps (sweeps per running job) per round
constexpr int kRoundsInFlight = 2;
constexpr int kTrajAhead = 2;
constexpr int kClasses = 3;  // Metropolis size classes (separate round streams)
// result slots in lat->s_out / lat->h_results
constexpr int kSlotPlaq = 0, kSlotHmc = 4, kSlotWilson = 8;  // wilson: kSlotWilson + mu * KLFT_JOB_MAX_WILSON + k
constexpr int kSlotsUsed = kSlotWilson + 3 * KLFT_JOB_MAX_WILSON;
static_assert(kSlotsUsed <= KLFT_RESULT_SLOTS, "result slots");

using Clock = std::chrono::steady_clock;

struct Job {
  uint64_t id = 0;
  klft_job d{};
  uint64_t footprint = 0;
  double t_submit = 0.0, t_admit = 0.0;
  std::atomic<bool> cancel{false};
  // worker-owned from admission on
  klft_lattice *lat = nullptr;
  int slot = -1;  // accept-counter index (Metropolis)
  int cls = 0;    // Metropolis size class
  int todo = 0;   // sweeps or trajectories not yet enqueued
  int issued = 0, done_traj = 0;
  bool finishing = false, canceled = false;
  cudaEvent_t ev = nullptr;      // completion of the job's last enqueued work
  cudaEvent_t tev[kTrajAhead] = {};
  cudaEvent_t last_round = nullptr;  // last round event that swept this job
  WilsonPlan plan;
};

double secs(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

long long job_volume(const klft_job &d) {
  long long V = 1;
  for (int i = 0; i < d.ndims; ++i) V *= d.L[i];
  return V;
}

int u_updates_per_traj(const klft_job &d) {
  if (d.integrator == KLFT_INTEGRATOR_REFERENCE_LEAPFROG) return d.nsteps + 1;
  if (d.integrator == KLFT_INTEGRATOR_LEAPFROG) return d.nsteps;
  return 2 * d.nsteps;
}

unsigned long long job_link_updates(const klft_job &d) {
  const unsigned long long links = (unsigned long long)job_volume(d) * (unsigned long long)d.ndims;
  if (d.kind == KLFT_JOB_METROPOLIS) return links * (unsigned long long)d.nsweeps;
  return links * (unsigned long long)d.ntraj * (unsigned long long)u_updates_per_traj(d);
}

bool finite(double x) { return std::isfinite(x); }

// Metropolis size class by the cost of one sweep: links x a per-group weight
// (U(1) 1, SU(2) 3, SU(3) 10), doubled for FP64.  Class 0 holds lattices whose
// sweeps are launch- and latency-bound, class 2 the ones that fill the GPU.
int size_class(const klft_job &d) {
  const double w = d.nc == 1 ? 1.0 : (d.nc == 2 ? 3.0 : 10.0);
  const double c = (double)job_volume(d) * d.ndims * w * (d.precision == KLFT_PRECISION_FP64 ? 2.0 : 1.0);
  return c < 1.0e6 ? 0 : (c < 8.0e6 ? 1 : 2);
}

klft_status validate(const klft_job *j) {
  if (!j) return fail(KLFT_EINVAL, "klft_server_submit: null job");
  if (j->kind != KLFT_JOB_METROPOLIS && j->kind != KLFT_JOB_HMC)
    return fail(KLFT_EINVAL, "job: unknown kind %d", j->kind);
  if (j->nc < 1 || j->nc > 3) return fail(KLFT_EINVAL, "job: Nc must be 1, 2 or 3 (got %d)", j->nc);
  if (j->ndims < 2 || j->ndims > 4) return fail(KLFT_EINVAL, "job: ndims must be 2, 3 or 4 (got %d)", j->ndims);
  long long V = 1;
  for (int d = 0; d < j->ndims; ++d) {
    if (j->L[d] < 2 || (j->L[d] & 1)) return fail(KLFT_EINVAL, "job: extent L%d = %d must be even and >= 2", d, j->L[d]);
    V *= j->L[d];
    if (V > 0x7fffffffLL) return fail(KLFT_EINVAL, "job: volume exceeds 2^31-1");
  }
  if (j->precision != KLFT_PRECISION_FP64 && j->precision != KLFT_PRECISION_MIXED)
    return fail(KLFT_EINVAL, "job: unknown precision %d", j->precision);
  if (j->start != KLFT_START_COLD && j->start != KLFT_START_HOT) return fail(KLFT_EINVAL, "job: unknown start %d", j->start);
  if (!finite(j->beta)) return fail(KLFT_EINVAL, "job: beta must be finite");
  if (j->kind == KLFT_JOB_METROPOLIS) {
    if (j->nsweeps < 0 || j->nhits < 0) return fail(KLFT_EINVAL, "job: negative sweep or hit count");
    if (j->proposal != KLFT_PROPOSAL_REFERENCE && j->proposal != KLFT_PROPOSAL_EXP)
      return fail(KLFT_EINVAL, "job: unknown proposal %d", j->proposal);
    if (!finite(j->delta) || !finite(j->eps)) return fail(KLFT_EINVAL, "job: step sizes must be finite");
    if (j->nc == 3 && j->proposal == KLFT_PROPOSAL_REFERENCE && !(j->delta > 0.0))
      return fail(KLFT_EINVAL, "job: the reference SU(3) proposal needs delta > 0");
  } else {
    if (j->ntraj < 0) return fail(KLFT_EINVAL, "job: negative trajectory count");
    if (j->nsteps < 1) return fail(KLFT_EINVAL, "job: n_steps must be >= 1");
    if (!finite(j->tau)) return fail(KLFT_EINVAL, "job: tau must be finite");
    if (j->integrator < KLFT_INTEGRATOR_REFERENCE_LEAPFROG || j->integrator > KLFT_INTEGRATOR_OMELYAN)
      return fail(KLFT_EINVAL, "job: unknown integrator %d", j->integrator);
  }
  if (j->n_wilson < 0 || j->n_wilson > KLFT_JOB_MAX_WILSON)
    return fail(KLFT_EINVAL, "job: n_wilson must be in 0..%d", KLFT_JOB_MAX_WILSON);
  for (int k = 0; k < 2 * j->n_wilson; ++k)
    if (j->wilson_pairs[k] < 0) return fail(KLFT_EINVAL, "job: negative loop extent");
  return KLFT_OK;
}

uint64_t footprint_of(const klft_job &j) {
  const Geom g = make_geom(j.ndims, j.L);
  const int dtype = j.precision == KLFT_PRECISION_FP64 ? 0 : 1;
  uint64_t b = (uint64_t)g.V * j.ndims * link_planes(j.nc, dtype) * (dtype == 0 ? 16 : 8);  // links
  b += 4096 + KLFT_RESULT_SLOTS * sizeof(double);                            // counters, result slots
  b += (uint64_t)plaquette_blocks(g) * sizeof(double);
  if (j.n_wilson > 0) {
    int tmax = 0;
    for (int k = 0; k < j.n_wilson; ++k) tmax = std::max(tmax, j.wilson_pairs[2 * k + 1]);
    b += wilson_gf_scratch(j.nc, dtype, g, j.ndims - 1, tmax, j.ndims - 1);
    b += (uint64_t)std::max(wilson_gf_blocks(g), plaquette_blocks(g)) * j.n_wilson * (j.ndims - 1) * sizeof(double) +
         4096;
  }
  if (j.kind == KLFT_JOB_HMC) b += hmc_footprint(j.nc, dtype, g, std::max(j.ntraj, 1));
  return b;
}

}  // namespace

struct klft_server {
  int device = 0;
  uint64_t budget = 0;
  int max_active = 256, max_queued = 4096;
  Clock::time_point t0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::unique_ptr<Job>> queue;
  std::unordered_map<uint64_t, Job *> live;  // queued or running
  std::deque<klft_job_result> done;
  uint64_t next_id = 1;
  bool stop = false;
  std::atomic<int> inject{0};
  // statistics (under mu), and the worker's own counters
  klft_server_stats st{};
  std::atomic<unsigned long long> launches{0}, nrounds{0};
  int running = 0;
  uint64_t in_use = 0;

  // worker-owned
  std::thread worker;
  cudaStream_t stream = nullptr;  // class 0 (and server-level work)
  cudaStream_t cls_stream[kClasses] = {};
  // per class: side streams for the second and later launch groups of a round
  // step (jobs of different Nc, Nd, precision or proposal share no data)
  static constexpr int kSide = 2;
  cudaStream_t side[kClasses][kSide] = {};
  cudaEvent_t ev_fork[kClasses] = {}, ev_join[kClasses][kSide] = {};
  void destroy_side() {
    for (int k = 0; k < kClasses; ++k) {
      for (int i = 0; i < kSide; ++i) {
        if (side[k][i]) cudaStreamDestroy(side[k][i]);
        if (ev_join[k][i]) cudaEventDestroy(ev_join[k][i]);
        side[k][i] = nullptr;
        ev_join[k][i] = nullptr;
      }
      if (ev_fork[k]) cudaEventDestroy(ev_fork[k]);
      ev_fork[k] = nullptr;
    }
  }
  unsigned long long *d_nacc = nullptr, *h_nacc = nullptr;
  uint32_t *d_zero = nullptr;
  std::vector<int> free_slots;
  std::vector<std::unique_ptr<Job>> jobs;  // running (admitted) jobs
  std::deque<cudaEvent_t> rounds[kClasses];  // in flight per class, oldest first
  std::vector<cudaEvent_t> event_pool;
  double busy_since = -1.0;

  void post(klft_job_result r) {
    std::lock_guard<std::mutex> g(mu);
    switch (r.status) {
      case KLFT_OK: st.completed++; st.link_updates += r.link_updates; break;
      case KLFT_ECANCELED: st.cancelled++; break;
      default: st.failed++;
    }
    done.push_back(r);
    cv_done.notify_all();
  }

  void run();
  bool step();
  void admit(std::unique_ptr<Job> j);
  void finish(Job &j, bool failed, int status, const char *msg);
  void fail_all(const char *msg);
  bool enqueue_round(int cls);
  void start_measure(Job &j, cudaEvent_t after);
  cudaEvent_t get_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) throw std::runtime_error("cudaEventCreate");
    return e;
  }
};

namespace {

klft_job_result base_result(const Job &j, double t_finish) {
  klft_job_result r;
  std::memset(&r, 0, sizeof r);
  r.id = j.id;
  r.kind = j.d.kind;
  r.plaquette = NAN;
  for (double &w : r.wilson) w = NAN;
  r.acceptance = NAN;
  r.mean_exp_mdH = NAN;
  r.mean_dH = NAN;
  r.t_submit = j.t_submit;
  r.t_admit = j.t_admit;
  r.t_finish = t_finish;
  return r;
}

void release_job(klft_server &s, Job &j) {
  for (cudaEvent_t &e : j.tev)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  if (j.ev) { cudaEventDestroy(j.ev); j.ev = nullptr; }
  if (j.lat) { klft_lattice_destroy(j.lat); j.lat = nullptr; }
  if (j.slot >= 0) { s.free_slots.push_back(j.slot); j.slot = -1; }
}

}  // namespace

// Called on the worker once a job's lattice exists or failed to exist.
void klft_server::admit(std::unique_ptr<Job> jp) {
  Job &j = *jp;
  j.t_admit = secs(t0);
  auto bail = [&](int code) {
    klft_job_result r = base_result(j, secs(t0));
    r.status = code;
    std::snprintf(r.error, sizeof r.error, "%s", klft_last_error());
    release_job(*this, j);
    {
      std::lock_guard<std::mutex> g(mu);
      live.erase(j.id);
      running--;
      in_use -= j.footprint;
    }
    post(r);
  };
  klft_status s = klft_lattice_create(j.d.nc, j.d.ndims, j.d.L, j.d.precision, j.d.start, j.d.seed, &j.lat);
  if (s == KLFT_OK) s = klft_lattice_set_stream(j.lat, j.d.seed, j.d.chain);
  if (s != KLFT_OK) return bail(s);
  klft_lattice *lat = j.lat;
  auto ck = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && s == KLFT_OK) s = cuda_fail(e, what);
  };
  ck(lat->s_out.ensure(KLFT_RESULT_SLOTS * sizeof(double)), "result slots");
  ck(lat->s_part.ensure((size_t)plaquette_blocks(lat->g) * sizeof(double)), "partials");
  ck(cudaEventCreateWithFlags(&j.ev, cudaEventDisableTiming), "cudaEventCreate");
  if (s == KLFT_OK && j.d.n_wilson > 0)
    s = make_wilson_plan(lat, j.d.wilson_pairs, j.d.n_wilson, j.d.ndims - 1, j.plan, 0, j.d.ndims - 1);
  if (s == KLFT_OK && j.d.kind == KLFT_JOB_HMC) {
    s = hmc_prepare(lat, std::max(j.d.ntraj, 1));
    for (cudaEvent_t &e : j.tev) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    j.todo = j.d.ntraj;
  }
  if (s == KLFT_OK && j.d.kind == KLFT_JOB_METROPOLIS) {
    if (free_slots.empty()) s = fail(KLFT_EINTERNAL, "serving: no accept-counter slot left");
    else {
      j.slot = free_slots.back();
      free_slots.pop_back();
      j.cls = size_class(j.d);
      ck(cudaMemsetAsync(d_nacc + j.slot, 0, sizeof(unsigned long long), cls_stream[j.cls]), "clear accept counter");
    }
    j.todo = j.d.nsweeps;
  }
  // the lattice was initialised on its own stream: later rounds on the class
  // stream must see it
  if (s == KLFT_OK) ck(cudaStreamSynchronize(lat->stream), "admission");
  if (s != KLFT_OK) return bail(s);
  jobs.push_back(std::move(jp));
  if (j.d.kind == KLFT_JOB_METROPOLIS && j.todo == 0) start_measure(j, nullptr);
}

// Enqueue the final measurements of job j on its stream (after event `after`
// when given), then record j.ev.
void klft_server::start_measure(Job &j, cudaEvent_t after) {
  klft_lattice *lat = j.lat;
  klft_status s = KLFT_OK;
  auto ck = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && s == KLFT_OK) s = cuda_fail(e, what);
  };
  if (after) ck(cudaStreamWaitEvent(lat->stream, after, 0), "cudaStreamWaitEvent");
  double *d_out = (double *)lat->s_out.ptr;
  if (!j.canceled) {
    if (s == KLFT_OK && j.d.measure_plaquette) {
      s = enqueue_plaquette(lat, kSlotPlaq);
      launches += 2;
    }
    if (s == KLFT_OK && j.d.n_wilson > 0) {
      s = enqueue_wilson_spatial(lat, j.plan, false, d_out + kSlotWilson, KLFT_JOB_MAX_WILSON);
      // omega, U' per plane, the loop kernel, the reductions (one launch when the
      // planes' sums are contiguous, i.e. the pair list fills its slots)
      launches += (j.d.ndims - 1) + 2 + (j.d.n_wilson == KLFT_JOB_MAX_WILSON ? 1 : j.d.ndims - 1);
    }
    if (s == KLFT_OK && j.d.kind == KLFT_JOB_HMC) {
      s = hmc_enqueue_summary(lat, j.d.ntraj, d_out + kSlotHmc);
      launches += 1;
    }
    if (j.d.kind == KLFT_JOB_METROPOLIS)
      ck(cudaMemcpyAsync(h_nacc + j.slot, d_nacc + j.slot, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                         lat->stream),
         "accept counter");
    ck(cudaMemcpyAsync(lat->h_results, d_out, kSlotsUsed * sizeof(double), cudaMemcpyDeviceToHost, lat->stream),
       "results");
  }
  ck(cudaEventRecord(j.ev, lat->stream), "cudaEventRecord");
  if (s != KLFT_OK) throw std::runtime_error(klft_last_error());
  j.finishing = true;
}

// Post the result of a job whose work has completed and free it.
void klft_server::finish(Job &j, bool failed, int status, const char *msg) {
  klft_job_result r = base_result(j, secs(t0));
  if (failed) {
    r.status = status;
    std::snprintf(r.error, sizeof r.error, "%s", msg);
  } else if (j.canceled) {
    r.status = KLFT_ECANCELED;
    std::snprintf(r.error, sizeof r.error, "cancelled");
  } else {
    const klft_lattice *lat = j.lat;
    const double *h = lat->h_results;
    r.status = KLFT_OK;
    if (j.d.measure_plaquette) r.plaquette = normalize_plaquette(lat, h[kSlotPlaq]);
    const int nd = j.d.ndims;
    for (int k = 0; k < j.d.n_wilson; ++k) {
      double acc = 0.0;
      for (int mu = 0; mu < nd - 1; ++mu) {
        const double w = normalize_wilson(lat, h[kSlotWilson + mu * KLFT_JOB_MAX_WILSON + k]);
        acc = mu == 0 ? w : acc + w;
      }
      r.wilson[k] = acc / (double)(nd - 1);
    }
    if (j.d.kind == KLFT_JOB_METROPOLIS) {
      const double norm = (double)job_volume(j.d) * nd * j.d.nhits * j.d.nsweeps;
      r.acceptance = norm > 0 ? (double)h_nacc[j.slot] / norm : 0.0;
    } else if (j.d.ntraj > 0) {
      r.acceptance = h[kSlotHmc] / j.d.ntraj;
      r.mean_exp_mdH = h[kSlotHmc + 1] / j.d.ntraj;
      r.mean_dH = h[kSlotHmc + 2] / j.d.ntraj;
    }
    r.link_updates = job_link_updates(j.d);
  }
  release_job(*this, j);
  {
    std::lock_guard<std::mutex> g(mu);
    live.erase(j.id);
    running--;
    in_use -= j.footprint;
  }
  post(r);
}

// One round: kSweepsPerRound steps; step k sweeps every Metropolis job with
// more than k sweeps left.  Returns false when no job needed a sweep.
bool klft_server::enqueue_round(int cls) {
  cudaStream_t stream = cls_stream[cls];
  std::vector<Job *> metro;
  for (auto &jp : jobs)
    if (jp->d.kind == KLFT_JOB_METROPOLIS && jp->cls == cls && !jp->finishing && jp->todo > 0)
      metro.push_back(jp.get());
  if (metro.empty()) return false;
  for (int k = 0; k < kSweepsPerRound; ++k) {
    std::vector<SweepItem> items;
    std::vector<uint32_t *> ctrs;
    for (Job *j : metro)
      if (j->todo > k) {
        const klft_job &d = j->d;
        items.push_back(SweepItem{j->lat, MetroArgs{d.beta, d.delta, d.eps, d.nhits, d.proposal, j->lat->seed,
                                                    j->lat->chain},
                                  j->lat->defect, j->slot});
        ctrs.push_back(j->lat->d_counters);
      }
    if (items.empty()) break;
    int nl = 0;
    const StreamFork fork{ev_fork[cls], side[cls], ev_join[cls], kSide};
    klft_status s = enqueue_multi_sweep(items, d_nacc, d_zero, stream, max_active, &nl, &fork);
    if (s != KLFT_OK) throw std::runtime_error(klft_last_error());
    cudaError_t e = launch_advance_list(ctrs, stream, &nl);
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    launches += nl;
  }
  cudaEvent_t ev = get_event();
  if (cudaEventRecord(ev, stream) != cudaSuccess) throw std::runtime_error("cudaEventRecord(round)");
  rounds[cls].push_back(ev);
  nrounds++;
  for (Job *j : metro) {
    j->todo -= std::min(j->todo, kSweepsPerRound);
    j->last_round = ev;
    if (j->todo == 0) start_measure(*j, ev);
  }
  return true;
}

// One pass of the worker; returns whether anything happened.
bool klft_server::step() {
  if (inject.exchange(0) == 1) throw std::runtime_error("injected worker fault");
  bool progress = false;
  // 1. admission (FIFO; the head waits until it fits)
  for (;;) {
    std::unique_ptr<Job> jp;
    {
      std::lock_guard<std::mutex> g(mu);
      if (queue.empty()) break;
      Job &h = *queue.front();
      if (running >= max_active || in_use + h.footprint > budget) break;
      jp = std::move(queue.front());
      queue.pop_front();
      running++;
      in_use += jp->footprint;
    }
    if (busy_since < 0) busy_since = secs(t0);
    admit(std::move(jp));
    progress = true;
  }
  // 2. retire completed rounds
  for (auto &rq : rounds)
    while (!rq.empty() && cudaEventQuery(rq.front()) == cudaSuccess) {
      event_pool.push_back(rq.front());
      rq.pop_front();
      progress = true;
    }
  // 3. cancellations of running jobs: stop scheduling, wait for their work in flight
  for (auto &jp : jobs) {
    Job &j = *jp;
    if (!j.finishing && j.cancel.load()) {
      j.canceled = true;
      cudaEvent_t after = nullptr;
      if (j.d.kind == KLFT_JOB_METROPOLIS) after = j.last_round;
      start_measure(j, after);  // records j.ev after the work in flight (no measurement)
      progress = true;
    }
  }
  // 4. HMC trajectories on the jobs' own streams
  for (auto &jp : jobs) {
    Job &j = *jp;
    if (j.d.kind != KLFT_JOB_HMC || j.finishing) continue;
    while (j.done_traj < j.issued && cudaEventQuery(j.tev[j.done_traj % kTrajAhead]) == cudaSuccess) j.done_traj++;
    while (j.todo > 0 && j.issued - j.done_traj < kTrajAhead) {
      klft_status s = hmc_enqueue_trajectory(j.lat, j.d.beta, j.d.tau, j.d.nsteps, j.d.integrator, j.issued);
      if (s != KLFT_OK) throw std::runtime_error(klft_last_error());
      if (cudaEventRecord(j.tev[j.issued % kTrajAhead], j.lat->stream) != cudaSuccess)
        throw std::runtime_error("cudaEventRecord(trajectory)");
      // momenta, 2x energies (4), integrator (force + update per step), reunitarise, accept, restore
      launches += 8 + 2 * (u_updates_per_traj(j.d) + 1);
      j.issued++;
      j.todo--;
      progress = true;
    }
    if (j.todo == 0) {
      start_measure(j, nullptr);
      progress = true;
    }
  }
  // 5. Metropolis rounds, one pipeline per size class
  for (int k = 0; k < kClasses; ++k)
    while ((int)rounds[k].size() < kRoundsInFlight && enqueue_round(k)) progress = true;
  // 6. completions
  for (size_t i = 0; i < jobs.size();) {
    Job &j = *jobs[i];
    if (j.finishing && cudaEventQuery(j.ev) == cudaSuccess) {
      finish(j, false, KLFT_OK, "");
      jobs.erase(jobs.begin() + (long)i);
      progress = true;
    } else {
      ++i;
    }
  }
  if (jobs.empty() && busy_since >= 0) {
    std::lock_guard<std::mutex> g(mu);
    if (queue.empty()) {
      st.busy_s += secs(t0) - busy_since;
      busy_since = -1.0;
    }
  }
  return progress;
}

// After an exception: wait for the device work of every running job, then fail them.
void klft_server::fail_all(const char *msg) {
  for (cudaStream_t cs : cls_stream) cudaStreamSynchronize(cs);
  for (auto &jp : jobs) {
    if (jp->lat) cudaStreamSynchronize(jp->lat->stream);
    finish(*jp, true, KLFT_EINTERNAL, msg);
  }
  jobs.clear();
  for (auto &rq : rounds) {
    for (cudaEvent_t e : rq) event_pool.push_back(e);
    rq.clear();
  }
  cudaGetLastError();
}

void klft_server::run() {
  cudaSetDevice(device);
  for (;;) {
    {
      std::unique_lock<std::mutex> g(mu);
      if (stop) break;
    }
    bool progress = false;
    try {
      progress = step();
    } catch (const std::exception &e) {
      std::string m = std::string("worker: ") + e.what();
      fail_all(m.c_str());
      progress = true;
    }
    if (!progress) {
      std::unique_lock<std::mutex> g(mu);
      if (stop) break;
      cv_work.wait_for(g, std::chrono::microseconds(100));
    }
  }
  // shutdown: wait for work in flight, free everything; queued jobs are dropped
  for (cudaStream_t cs : cls_stream) cudaStreamSynchronize(cs);
  for (auto &jp : jobs) {
    if (jp->lat) cudaStreamSynchronize(jp->lat->stream);
    release_job(*this, *jp);
  }
  jobs.clear();
}

extern "C" {

klft_status klft_job_footprint(const klft_job *job, uint64_t *bytes) {
  if (!bytes) return fail(KLFT_EINVAL, "klft_job_footprint: null pointer");
  klft_status s = validate(job);
  if (s != KLFT_OK) return s;
  *bytes = footprint_of(*job);
  return KLFT_OK;
}

klft_status klft_server_create(int device, uint64_t budget_bytes, int max_active, int max_queued,
                               klft_server **out) {
  if (!out) return fail(KLFT_EINVAL, "klft_server_create: null pointer");
  *out = nullptr;
  if (max_active < 0 || max_queued < 0) return fail(KLFT_EINVAL, "klft_server_create: negative limit");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(KLFT_ECUDA, "klft_server_create: no CUDA device available");
  if (device < 0 || device >= ndev) return fail(KLFT_EINVAL, "klft_server_create: no device %d", device);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  std::unique_ptr<klft_server> s(new klft_server());
  s->device = device;
  s->max_active = max_active ? max_active : 256;
  s->max_queued = max_queued ? max_queued : 4096;
  if (!budget_bytes) {
    size_t fr = 0, tot = 0;
    e = cudaMemGetInfo(&fr, &tot);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemGetInfo");
    budget_bytes = (uint64_t)(0.9 * (double)fr);
  }
  s->budget = budget_bytes;
  s->st.bytes_budget = budget_bytes;
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  s->cls_stream[0] = s->stream;
  for (int k = 1; k < kClasses && e == cudaSuccess; ++k)
    e = cudaStreamCreateWithFlags(&s->cls_stream[k], cudaStreamNonBlocking);
  for (int k = 0; k < kClasses && e == cudaSuccess; ++k) {
    e = cudaEventCreateWithFlags(&s->ev_fork[k], cudaEventDisableTiming);
    for (int i = 0; i < klft_server::kSide && e == cudaSuccess; ++i) {
      e = cudaStreamCreateWithFlags(&s->side[k][i], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_join[k][i], cudaEventDisableTiming);
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&s->d_nacc, (size_t)s->max_active * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_nacc, (size_t)s->max_active * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&s->d_zero, 16);
  if (e == cudaSuccess) e = cudaMemset(s->d_zero, 0, 16);
  if (e != cudaSuccess) {
    klft_status st = cuda_fail(e, "klft_server_create");
    if (s->d_nacc) cudaFree(s->d_nacc);
    if (s->h_nacc) cudaFreeHost(s->h_nacc);
    if (s->d_zero) cudaFree(s->d_zero);
    s->destroy_side();
    for (int k = 1; k < kClasses; ++k)
      if (s->cls_stream[k]) cudaStreamDestroy(s->cls_stream[k]);
    if (s->stream) cudaStreamDestroy(s->stream);
    cudaSetDevice(prev);
    return st;
  }
  for (int i = s->max_active - 1; i >= 0; --i) s->free_slots.push_back(i);
  s->t0 = Clock::now();
  klft_server *raw = s.release();
  raw->worker = std::thread([raw] { raw->run(); });
  cudaSetDevice(prev);
  *out = raw;
  return KLFT_OK;
}

klft_status klft_server_destroy(klft_server *s) {
  if (!s) return KLFT_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  for (auto &rq : s->rounds)
    for (cudaEvent_t e : rq) cudaEventDestroy(e);
  for (cudaEvent_t e : s->event_pool) cudaEventDestroy(e);
  if (s->d_nacc) cudaFree(s->d_nacc);
  if (s->h_nacc) cudaFreeHost(s->h_nacc);
  if (s->d_zero) cudaFree(s->d_zero);
  s->destroy_side();
  for (int k = 1; k < kClasses; ++k)
    if (s->cls_stream[k]) cudaStreamDestroy(s->cls_stream[k]);
  if (s->stream) cudaStreamDestroy(s->stream);
  cudaSetDevice(prev);
  delete s;
  return KLFT_OK;
}

klft_status klft_server_submit(klft_server *s, const klft_job *job, uint64_t *id) {
  if (!s) return fail(KLFT_EINVAL, "klft_server_submit: null server");
  klft_status v = validate(job);
  if (v != KLFT_OK) {
    std::lock_guard<std::mutex> g(s->mu);
    s->st.rejected++;
    return v;
  }
  std::unique_ptr<Job> j(new Job());
  j->d = *job;
  j->footprint = footprint_of(*job);
  std::lock_guard<std::mutex> g(s->mu);
  if (j->footprint > s->budget) {
    s->st.rejected++;
    return fail(KLFT_ENOMEM, "klft_server_submit: job needs %llu bytes, the budget is %llu",
                (unsigned long long)j->footprint, (unsigned long long)s->budget);
  }
  if ((int)s->queue.size() >= s->max_queued) {
    s->st.rejected++;
    return fail(KLFT_EBUSY, "klft_server_submit: %d jobs already queued", (int)s->queue.size());
  }
  j->id = s->next_id++;
  j->t_submit = secs(s->t0);
  if (id) *id = j->id;
  s->live[j->id] = j.get();
  s->queue.push_back(std::move(j));
  s->st.submitted++;
  s->cv_work.notify_all();
  return KLFT_OK;
}

klft_status klft_server_cancel(klft_server *s, uint64_t id) {
  if (!s) return fail(KLFT_EINVAL, "klft_server_cancel: null server");
  std::unique_lock<std::mutex> g(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return fail(KLFT_EINVAL, "klft_server_cancel: job %llu is not queued or running",
                                       (unsigned long long)id);
  Job *j = it->second;
  for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
    if (q->get() == j) {
      klft_job_result r = base_result(*j, secs(s->t0));
      r.status = KLFT_ECANCELED;
      std::snprintf(r.error, sizeof r.error, "cancelled while queued");
      s->live.erase(it);
      s->queue.erase(q);
      g.unlock();
      s->post(r);
      return KLFT_OK;
    }
  j->cancel.store(true);
  s->cv_work.notify_all();
  return KLFT_OK;
}

klft_status klft_server_poll(klft_server *s, klft_job_result *out, int max, int timeout_ms, int *n) {
  if (!s || !n || (max > 0 && !out)) return fail(KLFT_EINVAL, "klft_server_poll: null pointer");
  *n = 0;
  std::unique_lock<std::mutex> g(s->mu);
  if (s->done.empty() && timeout_ms > 0)
    s->cv_done.wait_for(g, std::chrono::milliseconds(timeout_ms), [s] { return !s->done.empty(); });
  while (*n < max && !s->done.empty()) {
    out[(*n)++] = s->done.front();
    s->done.pop_front();
  }
  return KLFT_OK;
}

klft_status klft_server_stats_get(klft_server *s, klft_server_stats *st) {
  if (!s || !st) return fail(KLFT_EINVAL, "klft_server_stats_get: null pointer");
  std::lock_guard<std::mutex> g(s->mu);
  *st = s->st;
  st->queued = (int)s->queue.size();
  st->active = s->running;
  st->bytes_in_use = s->in_use;
  st->bytes_budget = s->budget;
  st->launches = s->launches.load();
  st->rounds = s->nrounds.load();
  return KLFT_OK;
}

klft_status klft_server_inject_fault(klft_server *s, int what) {
  if (!s) return fail(KLFT_EINVAL, "klft_server_inject_fault: null server");
  if (what != 1) return fail(KLFT_EINVAL, "klft_server_inject_fault: unknown fault %d", what);
  s->inject.store(what);
  std::lock_guard<std::mutex> g(s->mu);
  s->cv_work.notify_all();
  return KLFT_OK;
}

}  // extern "C"
