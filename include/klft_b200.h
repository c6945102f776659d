/* klft_b200.h -- C ABI of libklft_b200.so, the B200 (sm_100a) implementation of
 * klft's lattice-gauge update-and-measure path.
 *
 * Conventions
 *  - Every entry point returns klft_status; on failure klft_last_error() gives a
 *    thread-local message.  No exception crosses the ABI.
 *  - Opaque handles own device memory and one CUDA stream each (a lattice
 *    measured by klft_run_cycles or klft_run_metropolis gains a second one on
 *    that call).  Calls on one handle are serialised by the library; distinct
 *    handles may be used from different threads.  Calls return after their
 *    device work has completed.
 *  - Host link buffers use the interchange layout
 *        U[(((site*Nd + mu)*Nc + i)*Nc + j)*2 + {0: re, 1: im}]   (double)
 *    with site = x0 + L0*(x1 + L1*(x2 + L2*x3)).
 *  - There is no CPU fallback: without a usable CUDA device every call that
 *    needs one fails with KLFT_ECUDA.
 *
 * Each declaration names the reference (aniketsen/klft) interface it replaces.
 */
#ifndef KLFT_B200_H
#define KLFT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  KLFT_OK = 0,
  KLFT_EINVAL = 1,   /* bad argument                        */
  KLFT_ENOMEM = 2,   /* device or host allocation failed    */
  KLFT_ECUDA = 3,    /* CUDA runtime error / no device      */
  KLFT_ETIMEOUT = 4, /* a bounded wait gave up (reserved: no
                      * kernel here waits on a flag or a peer) */
  KLFT_ENOTSUP = 5,  /* combination not supported           */
  KLFT_ECANCELED = 6, /* serving: the job was cancelled     */
  KLFT_EINTERNAL = 7, /* serving: the worker failed          */
  KLFT_EBUSY = 8      /* serving: admission queue is full    */
} klft_status;

typedef enum { KLFT_PRECISION_FP64 = 0, KLFT_PRECISION_MIXED = 1 } klft_precision;
typedef enum { KLFT_START_COLD = 0, KLFT_START_HOT = 1 } klft_start;
/* SU(3) proposal: the reference Gram-Schmidt generator (SUN.hpp:192-251),
 * U' = U r as in Metropolis.hpp:91, or U' = X U with X = exp(i eps H), H
 * hermitian traceless Gaussian; accepted X U products are reunitarised once
 * after the link's hits.  U(1)/SU(2) always use the reference generators
 * (SUN.hpp:163-189). */
typedef enum { KLFT_PROPOSAL_REFERENCE = 0, KLFT_PROPOSAL_EXP = 1 } klft_proposal;

typedef struct klft_lattice klft_lattice;

/* Thread-local description of the last failure on this thread. */
const char *klft_last_error(void);
/* Library version (major*10000 + minor*100 + patch). */
int klft_version(void);
/* Number of visible CUDA devices. */
klft_status klft_device_count(int *n);
/* Make `device` current for the calling thread; lattices created afterwards on
 * this thread live there (one process per GPU; the device choice of
 * Kokkos::initialize in the reference, lib/HMC_SU2.cpp:30). */
klft_status klft_set_device(int device);

/* Create a gauge field of SU(nc) (nc = 1: U(1)) links on an ndims-dimensional
 * periodic lattice with even extents L[0..ndims-1] on the current device.
 * Replaces deviceGaugeField{,3D,2D}<Nd,Nc> construction (GaugeField.hpp:30-141,
 * 241-344, 437-540) and the cold start of lib/Metropolis.cpp:79-81.
 * start = COLD: identity links; HOT: Haar-random links from seed. */
klft_status klft_lattice_create(int nc, int ndims, const int *L, int precision, int start, uint64_t seed,
                                klft_lattice **out);
klft_status klft_lattice_destroy(klft_lattice *lat);
klft_status klft_lattice_info(const klft_lattice *lat, int *nc, int *ndims, int *L, int *precision,
                              long long *volume);
/* Random stream identity: seed and chain key the Philox stream; the sweep and
 * trajectory counters are its step words (checkpoint = links + these). */
klft_status klft_lattice_set_stream(klft_lattice *lat, uint64_t seed, uint64_t chain);
klft_status klft_lattice_get_counters(klft_lattice *lat, uint32_t *sweep, uint32_t *trajectory);
klft_status klft_lattice_set_counters(klft_lattice *lat, uint32_t sweep, uint32_t trajectory);
/* Copy links from / to a host buffer in the interchange layout. */
klft_status klft_lattice_upload(klft_lattice *lat, const double *host);
klft_status klft_lattice_download(klft_lattice *lat, double *host);
/* Open boundary in direction mu (the intent of GaugeField.hpp:168-185 openBC<mu>,
 * whose body indexes past the lattice and does not compile): the links U_mu on
 * the slice x_mu = L_mu - 1 are set to zero and never updated, so every staple,
 * plaquette and Wilson loop through them vanishes; reunitarisation and the
 * unitarity check skip them.  Uploads re-zero them.  mu = -1 on a periodic
 * lattice is a no-op; an open direction cannot be closed again. */
klft_status klft_lattice_set_open_boundary(klft_lattice *lat, int mu);

/* nsweeps Metropolis sweeps; acc_out[k] = acceptance of sweep k normalised as
 * sweep_Metropolis does (Metropolis.hpp:118-178).  Replaces sweep_Metropolis. */
klft_status klft_metropolis_sweeps(klft_lattice *lat, double beta, double delta, int nhits, int proposal,
                                   double eps, int nsweeps, double *acc_out);

/* GaugePlaquette<rank,Nc>(g, normalize=true) (GaugePlaquette.hpp:89-135). */
klft_status klft_plaquette(klft_lattice *lat, double *out);
/* WilsonLoop_mu_nu (WilsonLoop.hpp:170-245): out[k] = W(mu, nu, pairs[2k], pairs[2k+1]). */
klft_status klft_wilson_loop_mu_nu(klft_lattice *lat, int mu, int nu, const int *pairs, int npairs, double *out);
/* WilsonLoop_temporal (WilsonLoop.hpp:250-304): out[k] = W_temp(L = pairs[2k], T = pairs[2k+1]). */
klft_status klft_wilson_loop_temporal(klft_lattice *lat, const int *pairs, int npairs, double *out);
/* stapleField (Gauge_Util.hpp:27-97), any ndims; out in the interchange layout. */
klft_status klft_staple_field(klft_lattice *lat, double *out);
/* max over links of ||U^dagger U - 1||_F. */
klft_status klft_unitarity(klft_lattice *lat, double *out);
/* restoreSUN on every link (SUN.hpp:256-340), in FP64 for both precisions. */
klft_status klft_reunitarize(klft_lattice *lat);

/* ncycles update-and-measure cycles enqueued back to back on the handle's stream,
 * as run_metropolis does them (Metropolis.hpp:204-218): one sweep, then (when
 * asked) GaugePlaquette and WilsonLoop_temporal over npairs (L, T) pairs.
 * With loops to measure, the plaquette and the loop kernels run on a second
 * stream of the handle (created on the first such call) beside the loops'
 * gauge transformation and the next sweep, ordered by events; the results are
 * those of the cycle order.  acc_out[c], plaq_out[c], w_out[c*npairs + k]
 * receive the results (each may be NULL); device_ms the CUDA-event time of the
 * whole sequence. */
klft_status klft_run_cycles(klft_lattice *lat, double beta, double delta, int nhits, int proposal, double eps,
                            int ncycles, int measure_plaquette, const int *temporal_pairs, int npairs,
                            double *acc_out, double *plaq_out, double *w_out, double *device_ms);

/* run_metropolis (Metropolis.hpp:180-223) with measureGaugeObservables
 * (GaugeObservable.hpp:64-127) enqueued on the handle's stream without host
 * round trips: nsweeps sweeps; after sweep `step` with interval > 0,
 * step % interval == 0 and step != 0 (so nmeas = (nsweeps - 1) / interval
 * measurements), the plaquette (when measure_plaquette), WilsonLoop_temporal
 * over ntemporal (L, T) pairs and WilsonLoop_mu_nu over every (mu, nu) of
 * `planes` (nplanes (mu, nu) pairs) over nplanar (Lmu, Lnu) pairs.
 * acc_out[nsweeps], plaq_out[nmeas], wtemp_out[nmeas * ntemporal],
 * wmunu_out[nmeas * nplanes * nplanar] (plane-major); each may be NULL.
 * device_ms: CUDA-event time of the whole run. */
klft_status klft_run_metropolis(klft_lattice *lat, double beta, double delta, int nhits, int proposal, double eps,
                                int nsweeps, int interval, int measure_plaquette, const int *temporal_pairs,
                                int ntemporal, const int *planes, int nplanes, const int *planar_pairs, int nplanar,
                                double *acc_out, double *plaq_out, double *wtemp_out, double *wmunu_out,
                                double *device_ms);

/* ---------------------------------------------------------------- HMC
 * Conventions of the reference (AdjointGroup.hpp), extended to SU(3) with the
 * Gell-Mann generators t_a: U <- exp(i dt sum_a p_a t_a) U (U(1): e^{i dt p};
 * SU(2): t_a = Pauli matrices), H = sum p^2/2 - (beta/Nc) sum_P Re Tr P,
 * force F_a = (beta/Nc) Im Tr(t_a U S).  Momenta host layout:
 * P[(site*Nd + mu)*ncomp + a], ncomp = 1, 3, 8 for U(1), SU(2), SU(3). */
typedef enum {
  KLFT_INTEGRATOR_REFERENCE_LEAPFROG = 0, /* Integrator.hpp:26-53: n_steps+1 gauge updates of tau/n_steps */
  KLFT_INTEGRATOR_LEAPFROG = 1,           /* standard n-step leapfrog of length tau */
  KLFT_INTEGRATOR_OMELYAN = 2             /* 2nd-order minimum norm (the LP_LEAPFROG slot, Integrator.hpp:10-13) */
} klft_integrator;

/* HMC::hmc_step (HMC.hpp:48-71), ntraj times: Gaussian momenta, integrate,
 * dH in FP64, accept/reject on the device (reject restores the links).
 * dH_out[k], accepted_out[k] per trajectory (either may be NULL). */
klft_status klft_hmc_trajectories(klft_lattice *lat, double beta, double tau, int n_steps, int integrator,
                                  int ntraj, double *dH_out, int *accepted_out);
/* Leapfrog::integrate (Integrator.hpp:22-54) from the current momenta, then
 * reunitarisation; no accept/reject. */
klft_status klft_hmc_integrate(klft_lattice *lat, double beta, double tau, int n_steps, int integrator);
/* HamiltonianField::randomize_momentum (HamiltonianField.hpp:50-59) from the
 * (trajectory, site, mu) stream. */
klft_status klft_hmc_refresh_momenta(klft_lattice *lat);
klft_status klft_hmc_set_momenta(klft_lattice *lat, const double *host);
klft_status klft_hmc_get_momenta(klft_lattice *lat, double *host);
/* GaugeMonomial::derivative (GaugeMonomial.hpp:27-37): (beta/Nc) Adj(U S) per link, momenta layout. */
klft_status klft_gauge_force(klft_lattice *lat, double beta, double *host_force);
/* HamiltonianField::kinetic_energy (HamiltonianField.hpp:40-48) and the gauge
 * monomial energy -(beta/Nc) sum_P Re Tr P (GaugeMonomial.hpp:19-25), FP64. */
klft_status klft_hmc_energies(klft_lattice *lat, double beta, double *kinetic, double *gauge_action);

/* Normalisation of the HMC generators of a lattice.  REFERENCE (the default)
 * is klft's: t_a = Pauli matrices for SU(2) (AdjointGroup.hpp:98-105), the
 * Gell-Mann matrices for SU(3), U(1) e^{i p}.  HALF uses t_a / 2 (the common
 * normalisation, Tr t_a t_b = delta_ab / 2): U <- exp(i dt sum_a p_a t_a / 2) U
 * and F_a = (beta/Nc) Im Tr(t_a U S) / 2, with the same N(0,1) momenta and
 * kinetic energy.  Its leapfrog/Omelyan step of length dt is the reference
 * step of length dt/2, so HALF with (tau, n_steps) is the REFERENCE
 * trajectory with (tau/2, n_steps); klft_gauge_force returns the HALF force.
 * Server jobs use REFERENCE. */
typedef enum { KLFT_GENERATORS_REFERENCE = 0, KLFT_GENERATORS_HALF = 1 } klft_generators;
klft_status klft_hmc_set_generators(klft_lattice *lat, int generators);

/* ---------------------------------------------------------------- PTBC
 * PTBCGaugeField set_defect / shift_defect (PTBCGaugeField.hpp:187-206): links
 * mu = 0 at x0 = 0 whose spatial coordinates lie in pos + [0, len) (periodic)
 * carry the factor c in the sweep (staples and dS).  len = 0 removes the defect.
 * pos has Nd-1 entries (directions 1..Nd-1). */
klft_status klft_lattice_set_defect(klft_lattice *lat, int len, const int *pos, double c);
/* out2[n-1] = sum over plaquettes with n defect links of -(beta/Nc) Re Tr U_P
 * (raw links), n = 1, 2: the only part of the action a swap changes. */
klft_status klft_ptbc_defect_sums(klft_lattice *lat, double beta, double *out2);
/* Replica swap (no counterpart in the reference, which defines the defect but
 * never swaps): for k = 0..nrep-2 the replicas holding labels k and k+1 exchange
 * labels with probability min(1, exp(-dS)), dS = sum_n (c_k^n - c_{k+1}^n)
 * (A_n(b) - A_n(a)).  label_of_rep is updated in place, accepted[k] receives the
 * decisions, and every replica's defect takes its new label's coefficient. */
klft_status klft_ptbc_swap(klft_lattice *const *reps, int nrep, const double *c_of_label, int *label_of_rep,
                           double beta, uint64_t seed, uint32_t cycle, int *accepted);
/* The swap decisions of klft_ptbc_swap from defect sums alone, on the host (no
 * device work): A[2r], A[2r+1] = out2 of klft_ptbc_defect_sums for replica r.
 * Same decisions and random stream as klft_ptbc_swap.  For replicas spread over
 * processes or GPUs: every rank computes its replicas' sums, the sums are
 * all-gathered (one FP64 pair per replica), and every rank calls this with the
 * same arguments, so all ranks agree on the new labels without moving links. */
klft_status klft_ptbc_swap_sums(const double *A, int nrep, const double *c_of_label, int *label_of_rep,
                                uint64_t seed, uint32_t cycle, int *accepted);
/* Coefficient c of an existing defect (EINVAL when the lattice has none). */
klft_status klft_lattice_set_defect_c(klft_lattice *lat, double c);

/* ---------------------------------------------------------------- batches
 * No counterpart in the reference (which runs one lattice per process): many
 * chains of any group, dimension, extents and precision, plus optional PTBC
 * replicas, advanced together.  One cycle = one Metropolis sweep of every chain
 * (reference sweep order per chain), then replica swap attempts, then (when
 * asked) the plaquette of every chain.  With use_graph the cycle is captured
 * once as a CUDA graph and replayed.  Results are identical to running each
 * chain alone with klft_metropolis_sweeps / klft_ptbc_swap.  Member lattices
 * must not be used by other calls while klft_batch_run runs. */
typedef struct klft_batch klft_batch;
klft_status klft_batch_create(klft_batch **out);
klft_status klft_batch_destroy(klft_batch *b);
/* Adds an existing lattice (owned by the caller) with its Metropolis parameters. */
klft_status klft_batch_add_chain(klft_batch *b, klft_lattice *lat, double beta, double delta, int nhits,
                                 int proposal, double eps, int *chain_id);
/* Marks nrep chains (each with a defect set) as PTBC replicas; replica r starts
 * with label r and coefficient c_of_label[r]; swaps use the (cycle, pair)
 * stream of swap_seed. */
klft_status klft_batch_set_ptbc(klft_batch *b, const int *chain_ids, int nrep, const double *c_of_label,
                                double beta, uint64_t swap_seed);
/* ncycles cycles: acc_out[c*nchains + i], plaq_out[c*nchains + i] (normalised as
 * GaugePlaquette), labels_out[c*nrep + r] (label of replica r after cycle c);
 * device_ms = CUDA-event time of the cycles.  Outputs may be NULL. */
klft_status klft_batch_run(klft_batch *b, int ncycles, int measure_plaquette, int use_graph, double *acc_out,
                           double *plaq_out, int *labels_out, double *device_ms);
/* accepted swaps per neighbouring label pair since klft_batch_set_ptbc (nrep-1 entries). */
klft_status klft_batch_swap_stats(klft_batch *b, unsigned long long *accepted_per_pair);

/* ---------------------------------------------------------------- tuner
 * tune_and_launch_for / readTuneCache / writeTuneCache (Tuner.hpp:73-358):
 * with enabled != 0 (KLFT_TUNING=1) the first launch of a kernel under a key
 * times the candidate launch shapes and keeps the fastest.  Cache file lines:
 * "<rank> <key> <v0> ... <v{rank-1}>".  Results never depend on the shape. */
klft_status klft_tuner_configure(int enabled, int verbosity);
klft_status klft_tuner_read_cache(const char *path);
klft_status klft_tuner_write_cache(const char *path);
/* values[0..rank-1] of a cached key; *rank = 0 when absent. */
klft_status klft_tuner_lookup(const char *key, int *values, int *rank);
klft_status klft_tuner_clear(void);

/* ---------------------------------------------------------------- checkpoints
 * No counterpart in the reference (it has no configuration I/O; measurements
 * live in host vectors until a run ends, GaugeObservable.hpp:40-44).  A
 * checkpoint holds the links (host interchange layout, complex128; the mixed
 * form's FP32 values convert exactly), the Philox stream (seed, chain), the
 * sweep/trajectory/cycle counters and the PTBC defect, with FNV-1a checksums of
 * header and payload.  Random numbers depend only on those, so a lattice read
 * back continues bit for bit where the written one stopped.  Writes go to
 * "<path>.tmp" and are renamed into place. */
klft_status klft_checkpoint_write(klft_lattice *lat, const char *path);
/* KLFT_EINVAL for a missing, foreign, truncated or corrupted file (checked
 * before any device work). */
klft_status klft_checkpoint_read(const char *path, klft_lattice **out);

/* ---------------------------------------------------------------- serving
 * No counterpart in the reference (its only drivers are the metropolis and hmc
 * binaries, Metropolis.hpp:113-223 and HMC.hpp:20-117, one run per process).
 * A server owns one worker thread on one GPU.  Jobs are queued by
 * klft_server_submit and admitted in arrival order while their device
 * footprint (klft_job_footprint) fits the memory budget and fewer than
 * max_active jobs run.  Admitted jobs keep their lattice and RNG counters
 * resident until they finish.  Metropolis jobs advance together: every round
 * sweeps each running job once per step in multi-chain launches (one per
 * parity class and group of lattices of one kind), so jobs that arrive while
 * others run join the next round.  HMC jobs run trajectories on their own
 * streams beside the rounds.  A finished job is measured on its final
 * configuration (plaquette, temporal Wilson loops) and its result is posted
 * for klft_server_poll.  A job's result depends only on its description: it
 * is the same, bit for bit, alone and in any mix. */
typedef enum { KLFT_JOB_METROPOLIS = 0, KLFT_JOB_HMC = 1 } klft_job_kind;
#define KLFT_JOB_MAX_WILSON 16
typedef struct klft_job {
  int kind;      /* klft_job_kind */
  int nc, ndims; /* group U(1)/SU(2)/SU(3), 2..4 dims */
  int L[4];      /* even extents */
  int precision, start;
  uint64_t seed, chain; /* Philox stream of the job */
  double beta;
  /* Metropolis (klft_metropolis_sweeps) */
  int nsweeps, nhits, proposal;
  double delta, eps;
  /* HMC (klft_hmc_trajectories) */
  int ntraj, nsteps, integrator;
  double tau;
  /* measurements of the final configuration */
  int measure_plaquette;
  int n_wilson;                            /* temporal loops, <= KLFT_JOB_MAX_WILSON */
  int wilson_pairs[2 * KLFT_JOB_MAX_WILSON]; /* (L, T) pairs */
} klft_job;

typedef struct klft_job_result {
  uint64_t id;
  int status;                        /* KLFT_OK or why the job failed */
  int kind;
  double plaquette;                  /* NaN unless measured */
  double wilson[KLFT_JOB_MAX_WILSON]; /* W_temp of the requested pairs */
  double acceptance;                 /* accepted hits / proposals, or accepted trajectories / ntraj */
  double mean_exp_mdH;               /* HMC: <exp(-dH)>; NaN for Metropolis */
  double mean_dH;                    /* HMC: <dH> */
  unsigned long long link_updates;   /* links visited: sweeps * V * Nd, or integrator link updates */
  double t_submit, t_admit, t_finish; /* seconds on the server's steady clock */
  char error[160];
} klft_job_result;

typedef struct klft_server_stats {
  unsigned long long submitted, completed, failed, cancelled, rejected;
  int queued, active;
  uint64_t bytes_in_use, bytes_budget;
  unsigned long long link_updates; /* of completed jobs */
  unsigned long long rounds;       /* Metropolis rounds enqueued */
  unsigned long long launches;     /* kernels the worker launched */
  double busy_s;                   /* seconds with at least one job admitted */
} klft_server_stats;

typedef struct klft_server klft_server;
/* device: CUDA ordinal.  budget_bytes: device memory the jobs may hold (0: 90%
 * of the free memory at creation).  max_active: running jobs (0: 256).
 * max_queued: waiting jobs before submit answers KLFT_EBUSY (0: 4096). */
klft_status klft_server_create(int device, uint64_t budget_bytes, int max_active, int max_queued,
                               klft_server **out);
/* Stops the worker after the GPU work in flight; unpolled results are dropped. */
klft_status klft_server_destroy(klft_server *s);
/* Device bytes a job holds while admitted. */
klft_status klft_job_footprint(const klft_job *job, uint64_t *bytes);
/* KLFT_EINVAL: malformed job; KLFT_ENOMEM: footprint above the budget (never
 * admissible); KLFT_EBUSY: queue full.  *id identifies the job's result. */
klft_status klft_server_submit(klft_server *s, const klft_job *job, uint64_t *id);
/* A queued job is dropped, a running one stops after its work in flight; both
 * post a result with status KLFT_ECANCELED.  KLFT_EINVAL for unknown or
 * finished ids. */
klft_status klft_server_cancel(klft_server *s, uint64_t id);
/* Up to max finished results, in completion order; waits up to timeout_ms for
 * the first one (0: no wait). */
klft_status klft_server_poll(klft_server *s, klft_job_result *out, int max, int timeout_ms, int *n);
klft_status klft_server_stats_get(klft_server *s, klft_server_stats *st);
/* Host-side fault injection for tests: 1 = the worker throws at its next
 * iteration (running jobs fail with KLFT_EINTERNAL, the worker carries on). */
klft_status klft_server_inject_fault(klft_server *s, int what);

/* No counterpart in the reference.  klft_metropolis_sweeps without any
 * allocation, for callers that cannot let the library allocate when they sweep:
 * an application whose device memory is already handed to its own pool (a late
 * cudaMalloc would fail) or a latency-critical loop that must not pay
 * cudaMalloc/cudaFree (which can synchronise the whole device).  Same kernels,
 * same random stream, same results as klft_metropolis_sweeps; the per-sweep
 * acceptance counters live in a fixed device array of KLFT_NOALLOC_MAX_SWEEPS
 * entries (8 KB, held on every GPU that loads the library until exit) instead
 * of handle scratch.  nsweeps above that limit is rejected with KLFT_EINVAL.
 * The lattice's device must be current.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  That first call (like the first launch of any
 * kernel) may also make the driver load the library's kernels, which can
 * allocate driver memory once: a warm-up call after creating the lattice makes
 * every later call allocation-free.  The tuner is not started from here; a
 * launch shape it already chose is used.  All calls on a device share the array: each call
 * clears the counters it uses, and because calls whose GPU work overlapped
 * would race on them, a call holds a per-device lock until its stream is done. */
#define KLFT_NOALLOC_MAX_SWEEPS 1024
klft_status klft_metropolis_sweeps_noalloc(klft_lattice *lat, double beta, double delta, int nhits, int proposal,
                                           double eps, int nsweeps, double *acc_out);

/* Diagnostic with no reference counterpart: measured CUDA-core FMA throughput
 * (dtype 0: FP64, 1: FP32) of the current device in TFLOP/s, the roofline
 * denominator of this library's SU(N) kernels. */
klft_status klft_peak_flops(int dtype, double *tflops);

/* Diagnostic with no reference counterpart: the error of the mixed form's
 * Metropolis action change on one configuration.  For every link of an FP64
 * SU(3) lattice and each of its nhits exp(i eps H) proposals of the current
 * sweep's stream, dS is formed twice with the same proposal: in FP64 from the
 * FP64 links, and in FP32 from the links as the mixed form stores them (two FP32
 * rows).  out[0] hits, out[1] mean and out[2] rms of d = dS32 - dS64, out[3]
 * max |d|, out[4] the slope sum(dS64 d) / sum(dS64^2) (a relative error of the
 * action change, i.e. of beta), out[5] the fraction of hits whose accept
 * decision differs with the hit's uniform.  The links are not changed. */
klft_status klft_exp_proposal_dS_error(klft_lattice *lat, double beta, double eps, int nhits, double *out);

#ifdef __cplusplus
}
#endif
#endif /* KLFT_B200_H */
