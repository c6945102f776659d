// klft.hpp -- C++ API of klft-b200, the drop-in for klft's host interface
// (include/klft.hpp, Metropolis_Params.hpp, GaugeObservable.hpp,
// InputParser.hpp, lib/Metropolis.cpp, lib/HMC_*.cpp).  Everything here runs on
// the C ABI of include/klft_b200.h; the structs keep the reference's field
// names and defaults.
#pragma once

#include <array>
#include <complex>
#include <cstddef>
#include <string>
#include <vector>

#include "../klft_b200.h"

namespace klft {

using real_t = double;
using index_t = int;

// Metropolis_Params.hpp:28-99 (struct defaults; the YAML parser has its own)
struct MetropolisParams {
  index_t Ndims = 4;
  index_t L0 = 4, L1 = 4, L2 = 4, L3 = 4;
  index_t nHits = 10;
  index_t nSweep = 1000;
  index_t seed = 1234;
  size_t Nd = 4;
  size_t Nc = 2;
  real_t beta = 1.0;
  real_t delta = 0.1;
  // additions, ignored by the reference parser (so old inputs keep their meaning)
  int precision = KLFT_PRECISION_FP64;  // "fp64" | "mixed"
  int proposal = KLFT_PROPOSAL_REFERENCE;  // "reference" | "exp" (SU(3) only)
  real_t eps = 0.0;                     // step of the exp(i eps H) proposal
  int start = KLFT_START_COLD;          // "cold" | "hot"
  void print() const;
};

// GaugeObservable.hpp:31-61
struct GaugeObservableParams {
  size_t measurement_interval = 0;
  bool measure_plaquette = false;
  bool measure_wilson_loop_temporal = false;
  bool measure_wilson_loop_mu_nu = false;
  std::vector<std::array<index_t, 2>> W_temp_L_T_pairs;
  std::vector<std::array<index_t, 2>> W_mu_nu_pairs;
  std::vector<std::array<index_t, 2>> W_Lmu_Lnu_pairs;
  std::vector<size_t> measurement_steps;
  std::vector<real_t> plaquette_measurements;
  std::vector<std::vector<std::array<real_t, 3>>> W_temp_measurements;
  std::vector<std::vector<std::array<real_t, 5>>> W_mu_nu_measurements;
  std::string plaquette_filename, W_temp_filename, W_mu_nu_filename;
  bool write_to_file = false;
};

// HMC_Params.hpp and the hmc binary's flags (hmc.cpp:8-72)
struct HMCParams {
  std::string gauge_group = "SU2";  // U1 | SU2 | SU3
  int ndim = 4;
  size_t LX = 8, LY = 8, LZ = 8, LT = 16;
  size_t n_traj = 1000;
  size_t n_steps = 50;
  real_t tau = 1.0;
  real_t beta = 2.0;
  size_t seed = 1234;
  std::string outfilename;
  int integrator = KLFT_INTEGRATOR_REFERENCE_LEAPFROG;
  int precision = KLFT_PRECISION_FP64;
  int generators = KLFT_GENERATORS_REFERENCE;  // klft_hmc_set_generators
};

// InputParser.hpp:33-125: false (and a message) when the block is missing or malformed
bool parseInputFile(const std::string &filename, MetropolisParams &p);
bool parseInputFile(const std::string &filename, GaugeObservableParams &p);
bool parseInputFile(const std::string &filename, HMCParams &p);

// GaugePlaquette.hpp:89-135, WilsonLoop.hpp:170-304 on a lattice handle
real_t GaugePlaquette(klft_lattice *g, bool normalize = true);
void WilsonLoop_mu_nu(klft_lattice *g, index_t mu, index_t nu, const std::vector<std::array<index_t, 2>> &pairs,
                      std::vector<std::array<real_t, 5>> &out);
void WilsonLoop_temporal(klft_lattice *g, const std::vector<std::array<index_t, 2>> &pairs,
                         std::vector<std::array<real_t, 3>> &out);
// GaugeVector.hpp:237-262 (legacy GaugeVector path): one Lmu x Lnu loop in the
// (mu, nu) plane, mu != nu; Normalize divides the Re Tr sum by V * Nc
real_t get_W_loop_mu_nu(klft_lattice *g, index_t mu, index_t nu, index_t Lmu, index_t Lnu, bool Normalize = true);
// Gauge_Util.hpp:27-97: the staple of every link (periodic), complex128
// [V][Nd][Nc][Nc], site = x0 + L0*(x1 + L1*(x2 + L2*x3)); empty on error
std::vector<std::complex<double>> stapleField(klft_lattice *g);
// Metropolis.hpp:118-178
real_t sweep_Metropolis(klft_lattice *g, const MetropolisParams &p);
// GaugeObservable.hpp:64-127 and :130-240
void measureGaugeObservables(klft_lattice *g, GaugeObservableParams &p, size_t step);
void flushAllGaugeObservables(const GaugeObservableParams &p, bool HEADER = true);
void clearAllGaugeObservables(GaugeObservableParams &p);
// Metropolis.hpp:180-223
int run_metropolis(klft_lattice *g, const MetropolisParams &mp, GaugeObservableParams &op);

// lib/Metropolis.cpp:36-166 (klft.hpp:6): parse, cold start, run, flush; env
// KLFT_VERBOSITY, KLFT_TUNING, KLFT_CACHE_FILE.  0 on success, -1 on error.
int Metropolis(const std::string &input_file);
// lib/HMC_SU2.cpp / HMC_U1.cpp: trajectories with per-trajectory output
int HMC(const HMCParams &p);

int verbosity();

}  // namespace klft
