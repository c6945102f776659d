// lib_host.cpp -- the C++ host side of klft-b200 (include/klft/klft.hpp):
// input parsing, the Metropolis and HMC drivers, measurement bookkeeping and
// output files, as the reference does them (InputParser.hpp,
// GaugeObservable.hpp, Metropolis.hpp:180-223, lib/Metropolis.cpp,
// lib/HMC_SU2.cpp).  Device work goes through the C ABI only.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/klft/klft.hpp"
#include "yaml_lite.hpp"

namespace klft {

static int g_verbosity = 0;
int verbosity() { return g_verbosity; }

static int env_int(const char *name, int fallback) {
  const char *v = std::getenv(name);
  return v ? std::atoi(v) : fallback;
}

void MetropolisParams::print() const {
  // Metropolis_Params.hpp:80-97
  if (g_verbosity > 0) {
    printf("Metropolis Parameters:\n");
    printf("General Parameters:\n");
    printf("Ndims: %d\n", Ndims);
    printf("L0: %d\n", L0);
    printf("L1: %d\n", L1);
    printf("L2: %d\n", L2);
    printf("L3: %d\n", L3);
    printf("nHits: %d\n", nHits);
    printf("nSweep: %d\n", nSweep);
    printf("seed: %d\n", seed);
    printf("GaugeField Parameters:\n");
    printf("Nd: %zu\n", Nd);
    printf("Nc: %zu\n", Nc);
    printf("Wilson Action Parameters:\n");
    printf("beta: %.4f\n", beta);
    printf("delta: %.4f\n", delta);
  }
}

static int parse_choice(const yaml::Node &n, const char *a, int va, const char *b, int vb, int fallback) {
  if (!n) return fallback;
  const std::string s = n.as<std::string>("");
  if (s == a) return va;
  if (s == b) return vb;
  throw std::runtime_error(std::string("unknown value '") + s + "'");
}

// InputParser.hpp:33-66 (defaults L* = 32, nHits = 10, nSweep = 1000, seed = 1234,
// Nd = 4, Nc = 2, beta = 1.0, delta = 0.1)
bool parseInputFile(const std::string &filename, MetropolisParams &p) {
  try {
    const yaml::Node config = yaml::LoadFile(filename);
    if (config["MetropolisParams"]) {
      const yaml::Node &mp = config["MetropolisParams"];
      p.Ndims = mp["Ndims"].as<int>(4);
      p.L0 = mp["L0"].as<int>(32);
      p.L1 = mp["L1"].as<int>(32);
      p.L2 = mp["L2"].as<int>(32);
      p.L3 = mp["L3"].as<int>(32);
      p.nHits = mp["nHits"].as<int>(10);
      p.nSweep = mp["nSweep"].as<int>(1000);
      p.seed = mp["seed"].as<int>(1234);
      p.Nd = mp["Nd"].as<size_t>(4);
      p.Nc = mp["Nc"].as<size_t>(2);
      p.beta = mp["beta"].as<double>(1.0);
      p.delta = mp["delta"].as<double>(0.1);
      p.precision = parse_choice(mp["precision"], "fp64", KLFT_PRECISION_FP64, "mixed", KLFT_PRECISION_MIXED,
                                 KLFT_PRECISION_FP64);
      p.proposal = parse_choice(mp["proposal"], "reference", KLFT_PROPOSAL_REFERENCE, "exp", KLFT_PROPOSAL_EXP,
                                KLFT_PROPOSAL_REFERENCE);
      p.eps = mp["eps"].as<double>(0.0);
      p.start = parse_choice(mp["start"], "cold", KLFT_START_COLD, "hot", KLFT_START_HOT, KLFT_START_COLD);
    } else {
      printf("Error: MetropolisParams not found in input file\n");
      return false;
    }
    return true;
  } catch (const std::exception &e) {
    printf("Error parsing input file: %s\n", e.what());
    return false;
  }
}

static void read_pairs(const yaml::Node &n, std::vector<std::array<index_t, 2>> &out) {
  if (!n) return;
  for (const auto &pair : n) out.push_back({pair[0].as<int>(), pair[1].as<int>()});
}

// InputParser.hpp:69-125
bool parseInputFile(const std::string &filename, GaugeObservableParams &p) {
  try {
    const yaml::Node config = yaml::LoadFile(filename);
    if (config["GaugeObservableParams"]) {
      const yaml::Node &gp = config["GaugeObservableParams"];
      p.measurement_interval = gp["measurement_interval"].as<size_t>(0);
      p.measure_plaquette = gp["measure_plaquette"].as<bool>(false);
      p.measure_wilson_loop_temporal = gp["measure_wilson_loop_temporal"].as<bool>(false);
      p.measure_wilson_loop_mu_nu = gp["measure_wilson_loop_mu_nu"].as<bool>(false);
      read_pairs(gp["W_temp_L_T_pairs"], p.W_temp_L_T_pairs);
      read_pairs(gp["W_mu_nu_pairs"], p.W_mu_nu_pairs);
      read_pairs(gp["W_Lmu_Lnu_pairs"], p.W_Lmu_Lnu_pairs);
      p.plaquette_filename = gp["plaquette_filename"].as<std::string>("");
      p.W_temp_filename = gp["W_temp_filename"].as<std::string>("");
      p.W_mu_nu_filename = gp["W_mu_nu_filename"].as<std::string>("");
      p.write_to_file = gp["write_to_file"].as<bool>(false);
    } else {
      printf("Error: GaugeObservableParams not found in input file\n");
      return false;
    }
    return true;
  } catch (const std::exception &e) {
    printf("Error parsing input file: %s\n", e.what());
    return false;
  }
}

// An HMCParams block mirrors the hmc binary's flags (hmc.cpp:8-72)
bool parseInputFile(const std::string &filename, HMCParams &p) {
  try {
    const yaml::Node config = yaml::LoadFile(filename);
    if (!config["HMCParams"]) {
      printf("Error: HMCParams not found in input file\n");
      return false;
    }
    const yaml::Node &h = config["HMCParams"];
    p.gauge_group = h["gauge_group"].as<std::string>(p.gauge_group);
    p.ndim = h["ndim"].as<int>(p.ndim);
    p.LX = h["LX"].as<size_t>(p.LX);
    p.LY = h["LY"].as<size_t>(p.LY);
    p.LZ = h["LZ"].as<size_t>(p.LZ);
    p.LT = h["LT"].as<size_t>(p.LT);
    p.n_traj = h["n_traj"].as<size_t>(p.n_traj);
    p.n_steps = h["n_steps"].as<size_t>(p.n_steps);
    p.tau = h["tau"].as<double>(p.tau);
    p.beta = h["beta"].as<double>(p.beta);
    p.seed = h["seed"].as<size_t>(p.seed);
    p.outfilename = h["outfilename"].as<std::string>(p.outfilename);
    if (h["integrator"]) {
      const std::string s = h["integrator"].as<std::string>("");
      if (s == "reference") p.integrator = KLFT_INTEGRATOR_REFERENCE_LEAPFROG;
      else if (s == "leapfrog") p.integrator = KLFT_INTEGRATOR_LEAPFROG;
      else if (s == "omelyan") p.integrator = KLFT_INTEGRATOR_OMELYAN;
      else throw std::runtime_error("unknown integrator '" + s + "'");
    }
    p.precision = parse_choice(h["precision"], "fp64", KLFT_PRECISION_FP64, "mixed", KLFT_PRECISION_MIXED,
                               p.precision);
    p.generators = parse_choice(h["generators"], "reference", KLFT_GENERATORS_REFERENCE, "half",
                                KLFT_GENERATORS_HALF, p.generators);
    return true;
  } catch (const std::exception &e) {
    printf("Error parsing input file: %s\n", e.what());
    return false;
  }
}

static void report(klft_status s, const char *what) {
  if (s != KLFT_OK) fprintf(stderr, "%s: %s\n", what, klft_last_error());
}

real_t GaugePlaquette(klft_lattice *g, bool normalize) {
  double P = 0.0;
  report(klft_plaquette(g, &P), "GaugePlaquette");
  if (!normalize) {
    int nc = 0, nd = 0;
    long long V = 0;
    klft_lattice_info(g, &nc, &nd, nullptr, nullptr, &V);
    P *= (double)V * (double)((nd * (nd - 1) / 2) * nc);
  }
  return P;
}

static std::vector<int> flat(const std::vector<std::array<index_t, 2>> &pairs) {
  std::vector<int> f;
  for (const auto &p : pairs) {
    f.push_back(p[0]);
    f.push_back(p[1]);
  }
  return f;
}

void WilsonLoop_mu_nu(klft_lattice *g, index_t mu, index_t nu, const std::vector<std::array<index_t, 2>> &pairs,
                      std::vector<std::array<real_t, 5>> &out) {
  if (pairs.empty()) return;
  const std::vector<int> f = flat(pairs);
  std::vector<double> w(pairs.size());
  report(klft_wilson_loop_mu_nu(g, mu, nu, f.data(), (int)pairs.size(), w.data()), "WilsonLoop_mu_nu");
  for (size_t k = 0; k < pairs.size(); ++k)
    out.push_back({(real_t)mu, (real_t)nu, (real_t)pairs[k][0], (real_t)pairs[k][1], w[k]});
}

void WilsonLoop_temporal(klft_lattice *g, const std::vector<std::array<index_t, 2>> &pairs,
                         std::vector<std::array<real_t, 3>> &out) {
  if (pairs.empty()) return;
  const std::vector<int> f = flat(pairs);
  std::vector<double> w(pairs.size());
  report(klft_wilson_loop_temporal(g, f.data(), (int)pairs.size(), w.data()), "WilsonLoop_temporal");
  for (size_t k = 0; k < pairs.size(); ++k) out.push_back({(real_t)pairs[k][0], (real_t)pairs[k][1], w[k]});
}

real_t get_W_loop_mu_nu(klft_lattice *g, index_t mu, index_t nu, index_t Lmu, index_t Lnu, bool Normalize) {
  const int pair[2] = {Lmu, Lnu};
  double w = 0.0;
  report(klft_wilson_loop_mu_nu(g, mu, nu, pair, 1, &w), "get_W_loop_mu_nu");
  if (!Normalize) {
    int nc = 0, nd = 0;
    long long V = 0;
    klft_lattice_info(g, &nc, &nd, nullptr, nullptr, &V);
    w *= (double)V * (double)nc;
  }
  return w;
}

std::vector<std::complex<double>> stapleField(klft_lattice *g) {
  int nc = 0, nd = 0;
  long long V = 0;
  report(klft_lattice_info(g, &nc, &nd, nullptr, nullptr, &V), "stapleField");
  std::vector<std::complex<double>> out((size_t)V * nd * nc * nc);
  const klft_status s = klft_staple_field(g, reinterpret_cast<double *>(out.data()));
  report(s, "stapleField");
  if (s != KLFT_OK) out.clear();
  return out;
}

real_t sweep_Metropolis(klft_lattice *g, const MetropolisParams &p) {
  double acc = 0.0;
  report(klft_metropolis_sweeps(g, p.beta, p.delta, p.nHits, p.proposal, p.eps, 1, &acc), "sweep_Metropolis");
  return acc;
}

// GaugeObservable.hpp:64-127
void measureGaugeObservables(klft_lattice *g, GaugeObservableParams &params, size_t step) {
  if ((params.measurement_interval == 0) || (step % params.measurement_interval != 0) || (step == 0)) return;
  if (g_verbosity > 0) {
    printf("Measurement of Gauge Observables\n");
    printf("step: %zu\n", step);
  }
  if (params.measure_plaquette) {
    const real_t P = GaugePlaquette(g);
    params.plaquette_measurements.push_back(P);
    if (g_verbosity > 0) printf("plaquette: %11.6f\n", P);
  }
  if (params.measure_wilson_loop_temporal) {
    if (g_verbosity > 0) {
      printf("temporal Wilson loop:\n");
      printf("L, T, W_temp\n");
    }
    std::vector<std::array<real_t, 3>> temp;
    WilsonLoop_temporal(g, params.W_temp_L_T_pairs, temp);
    if (g_verbosity > 0)
      for (const auto &m : temp) printf("%d, %d, %11.6f\n", (index_t)m[0], (index_t)m[1], m[2]);
    params.W_temp_measurements.push_back(temp);
  }
  if (params.measure_wilson_loop_mu_nu) {
    if (g_verbosity > 0) {
      printf("Wilson loop in the mu-nu plane:\n");
      printf("mu, nu, Lmu, Lnu, W_mu_nu\n");
    }
    std::vector<std::array<real_t, 5>> temp;
    for (const auto &mn : params.W_mu_nu_pairs) {
      WilsonLoop_mu_nu(g, mn[0], mn[1], params.W_Lmu_Lnu_pairs, temp);
      if (g_verbosity > 0)
        for (const auto &m : temp)
          printf("%d, %d, %d, %d, %11.6f\n", (index_t)m[0], (index_t)m[1], (index_t)m[2], (index_t)m[3], m[4]);
    }
    params.W_mu_nu_measurements.push_back(temp);
  }
  params.measurement_steps.push_back(step);
}

// GaugeObservable.hpp:130-230: append, default ostream formatting
void flushAllGaugeObservables(const GaugeObservableParams &params, bool HEADER) {
  if (!params.write_to_file) {
    printf("write_to_file is not enabled\n");
    return;
  }
  if (params.plaquette_filename != "") {
    std::ofstream file(params.plaquette_filename, std::ios::app);
    if (!file.is_open()) {
      printf("Error: file is not open\n");
    } else if (!params.measure_plaquette) {
      printf("Error: no plaquette measurements available\n");
    } else {
      if (HEADER) file << "# step, plaquette\n";
      for (size_t i = 0; i < params.measurement_steps.size(); ++i)
        file << params.measurement_steps[i] << ", " << params.plaquette_measurements[i] << "\n";
    }
  }
  if (params.W_temp_filename != "") {
    std::ofstream file(params.W_temp_filename, std::ios::app);
    if (!file.is_open()) {
      printf("Error: file is not open\n");
    } else if (!params.measure_wilson_loop_temporal) {
      printf("Error: no temporal Wilson loop measurements available\n");
    } else {
      if (HEADER) file << "# step, L, T, W_temp\n";
      for (size_t i = 0; i < params.measurement_steps.size(); ++i)
        for (const auto &m : params.W_temp_measurements[i])
          file << params.measurement_steps[i] << ", " << m[0] << ", " << m[1] << ", " << m[2] << "\n";
    }
  }
  if (params.W_mu_nu_filename != "") {
    std::ofstream file(params.W_mu_nu_filename, std::ios::app);
    if (!file.is_open()) {
      printf("Error: file is not open\n");
    } else if (!params.measure_wilson_loop_mu_nu) {
      printf("Error: no mu-nu Wilson loop measurements available\n");
    } else {
      if (HEADER) file << "# step, mu, nu, Lmu, Lnu, W_mu_nu\n";
      for (size_t i = 0; i < params.measurement_steps.size(); ++i)
        for (const auto &m : params.W_mu_nu_measurements[i])
          file << params.measurement_steps[i] << ", " << m[0] << ", " << m[1] << ", " << m[2] << ", " << m[3] << ", "
               << m[4] << "\n";
    }
  }
}

void clearAllGaugeObservables(GaugeObservableParams &p) {
  p.measurement_steps.clear();
  p.plaquette_measurements.clear();
  p.W_temp_measurements.clear();
  p.W_mu_nu_measurements.clear();
}

// Metropolis.hpp:180-223
// Without per-step output the whole loop is one klft_run_metropolis call (the
// same sweeps and measurements, no host round trip per step).
static int run_metropolis_fused(klft_lattice *g, const MetropolisParams &mp, GaugeObservableParams &op) {
  std::vector<int> tp, pl, pp;
  if (op.measure_wilson_loop_temporal)
    for (const auto &q : op.W_temp_L_T_pairs) { tp.push_back(q[0]); tp.push_back(q[1]); }
  if (op.measure_wilson_loop_mu_nu) {
    for (const auto &q : op.W_mu_nu_pairs) { pl.push_back(q[0]); pl.push_back(q[1]); }
    for (const auto &q : op.W_Lmu_Lnu_pairs) { pp.push_back(q[0]); pp.push_back(q[1]); }
  }
  const int nsweeps = (int)mp.nSweep, interval = (int)op.measurement_interval;
  const int nmeas = interval > 0 && nsweeps > 0 ? (nsweeps - 1) / interval : 0;
  const int ntp = (int)tp.size() / 2, npl = (int)pl.size() / 2, npp = (int)pp.size() / 2;
  std::vector<double> plaq(nmeas > 0 ? nmeas : 1), wt((size_t)(nmeas > 0 ? nmeas : 1) * (ntp > 0 ? ntp : 1)),
      wm((size_t)(nmeas > 0 ? nmeas : 1) * (npl * npp > 0 ? npl * npp : 1));
  if (klft_run_metropolis(g, mp.beta, mp.delta, (int)mp.nHits, mp.proposal, mp.eps, nsweeps, interval,
                          op.measure_plaquette ? 1 : 0, tp.data(), ntp, pl.data(), npl, pp.data(), npp, nullptr,
                          plaq.data(), wt.data(), wm.data(), nullptr) != KLFT_OK) {
    printf("Error: %s\n", klft_last_error());
    return -1;
  }
  for (int i = 0; i < nmeas; ++i) {
    if (op.measure_plaquette) op.plaquette_measurements.push_back(plaq[i]);
    if (op.measure_wilson_loop_temporal) {
      std::vector<std::array<real_t, 3>> rows;
      for (int k = 0; k < ntp; ++k) rows.push_back({(real_t)tp[2 * k], (real_t)tp[2 * k + 1], wt[(size_t)i * ntp + k]});
      op.W_temp_measurements.push_back(rows);
    }
    if (op.measure_wilson_loop_mu_nu) {
      std::vector<std::array<real_t, 5>> rows;
      for (int q = 0; q < npl; ++q)
        for (int k = 0; k < npp; ++k)
          rows.push_back({(real_t)pl[2 * q], (real_t)pl[2 * q + 1], (real_t)pp[2 * k], (real_t)pp[2 * k + 1],
                          wm[((size_t)i * npl + q) * npp + k]});
      op.W_mu_nu_measurements.push_back(rows);
    }
    op.measurement_steps.push_back((size_t)(i + 1) * op.measurement_interval);
  }
  flushAllGaugeObservables(op);
  return 0;
}

int run_metropolis(klft_lattice *g, const MetropolisParams &mp, GaugeObservableParams &op) {
  if (g_verbosity == 0) return run_metropolis_fused(g, mp, op);
  for (size_t step = 0; step < (size_t)mp.nSweep; ++step) {
    const auto t0 = std::chrono::steady_clock::now();
    const real_t acc_rate = sweep_Metropolis(g, mp);
    const double time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (g_verbosity > 0) printf("Step: %ld, Acceptance rate: %f, Time: %f\n", (long)step, acc_rate, time);
    measureGaugeObservables(g, op, step);
  }
  flushAllGaugeObservables(op);
  return 0;
}

static void tuning_from_env(bool start) {
  const int tuning = env_int("KLFT_TUNING", 0);
  const char *cache = std::getenv("KLFT_CACHE_FILE");
  if (start) {
    klft_tuner_configure(tuning, g_verbosity);
    if (tuning && cache) {
      if (g_verbosity > 0) printf("Reading cache file: %s\n", cache);
      klft_tuner_read_cache(cache);
    }
  } else if (tuning) {
    if (cache) klft_tuner_write_cache(cache);
    else printf("KLFT_CACHE_FILE not set\n");
  }
}

// lib/Metropolis.cpp:36-166
int Metropolis(const std::string &input_file) {
  g_verbosity = env_int("KLFT_VERBOSITY", 0);
  tuning_from_env(true);
  MetropolisParams mp;
  GaugeObservableParams op;
  if (!parseInputFile(input_file, mp)) {
    printf("Error parsing input file\n");
    return -1;
  }
  if (!parseInputFile(input_file, op)) {
    printf("Error parsing input file\n");
    return -1;
  }
  mp.print();
  if (mp.Ndims < 2 || mp.Ndims > 4 || (size_t)mp.Ndims != mp.Nd) {
    printf("Error: Unsupported dimensions\n");
    return -1;
  }
  if (mp.Nc < 1 || mp.Nc > 3) {
    printf("Error: Unsupported gauge group\n");
    return -1;
  }
  const int L[4] = {mp.L0, mp.L1, mp.L2, mp.L3};
  klft_lattice *g = nullptr;
  if (klft_lattice_create((int)mp.Nc, mp.Ndims, L, mp.precision, mp.start, (uint64_t)mp.seed, &g) != KLFT_OK) {
    printf("Error: %s\n", klft_last_error());
    return -1;
  }
  const int rc = run_metropolis(g, mp, op);
  klft_lattice_destroy(g);
  tuning_from_env(false);
  return rc;
}

// lib/HMC_SU2.cpp:9-75 (and the U(1) twin): banner, trajectories, per-trajectory line
int HMC(const HMCParams &p) {
  g_verbosity = env_int("KLFT_VERBOSITY", 0);
  tuning_from_env(true);
  const int nc = p.gauge_group == "U1" ? 1 : p.gauge_group == "SU2" ? 2 : p.gauge_group == "SU3" ? 3 : 0;
  if (!nc || p.ndim < 2 || p.ndim > 4) {
    printf("Error: unsupported gauge group %s / ndim %d\n", p.gauge_group.c_str(), p.ndim);
    return -1;
  }
  int L[4];
  if (p.ndim == 4) { L[0] = (int)p.LX; L[1] = (int)p.LY; L[2] = (int)p.LZ; L[3] = (int)p.LT; }
  else if (p.ndim == 3) { L[0] = (int)p.LX; L[1] = (int)p.LY; L[2] = (int)p.LT; L[3] = 1; }
  else { L[0] = (int)p.LX; L[1] = (int)p.LT; L[2] = L[3] = 1; }
  std::cout << "Running HMC_" << p.gauge_group << "_" << p.ndim << "D" << std::endl;
  std::cout << "HMC Parameters:" << std::endl;
  std::cout << "beta = " << p.beta << std::endl;
  std::cout << "n_traj = " << p.n_traj << std::endl;
  std::cout << "tau = " << p.tau << std::endl;
  std::cout << "n_steps = " << p.n_steps << std::endl;
  std::cout << "seed = " << p.seed << std::endl;
  std::cout << "output file = " << p.outfilename << std::endl;
  std::ofstream outfile;
  if (p.outfilename != "") {
    outfile.open(p.outfilename);
    outfile << "traj, accept, plaquette, time, acceptance rate" << std::endl;
  }
  klft_lattice *g = nullptr;
  if (klft_lattice_create(nc, p.ndim, L, p.precision, KLFT_START_HOT, (uint64_t)p.seed, &g) != KLFT_OK) {
    printf("Error: %s\n", klft_last_error());
    return -1;
  }
  klft_lattice_set_stream(g, (uint64_t)p.seed, 0);
  if (klft_hmc_set_generators(g, p.generators) != KLFT_OK) {
    printf("Error: %s\n", klft_last_error());
    klft_lattice_destroy(g);
    return -1;
  }
  double plaq = GaugePlaquette(g);
  std::cout << "Starting Plaquette: " << plaq << std::endl;
  std::cout << "Starting HMC: " << std::endl;
  size_t n_accept = 0;
  const auto t_all = std::chrono::steady_clock::now();
  for (size_t i = 0; i < p.n_traj; ++i) {
    const auto t0 = std::chrono::steady_clock::now();
    double dH = 0.0;
    int accept = 0;
    klft_status s = klft_hmc_trajectories(g, p.beta, p.tau, (int)p.n_steps, p.integrator, 1, &dH, &accept);
    if (s != KLFT_OK) {
      printf("Error: %s\n", klft_last_error());
      klft_lattice_destroy(g);
      return -1;
    }
    const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (accept) n_accept++;
    plaq = GaugePlaquette(g);
    std::cout << "Traj: " << i << " Accept: " << accept << " Plaquette: " << plaq << " Time: " << t
              << " Acceptance Rate: " << double(n_accept) / double(i + 1) << std::endl;
    if (p.outfilename != "")
      outfile << i << ", " << accept << ", " << plaq << ", " << t << ", " << double(n_accept) / double(i + 1)
              << std::endl;
  }
  std::cout << "HMC Time: " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t_all).count()
            << std::endl;
  klft_lattice_destroy(g);
  tuning_from_env(false);
  return 0;
}

}  // namespace klft
