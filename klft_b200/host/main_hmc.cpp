// hmc -- the klft `hmc` driver (hmc.cpp:6-80) on libklft_b200.  Same flags
// (--gauge-group U1|SU2 and now SU3, --ndim, --LX, --LY, --LZ, --LT, --n-traj,
// --n-steps, --tau, --beta, --seed, --outfilename, --help), plus
// --integrator reference|leapfrog|omelyan, --precision fp64|mixed,
// --generators reference|half (klft_hmc_set_generators) and -f <yaml> with an
// HMCParams block.
#include <cstdio>
#include <iostream>
#include <string>

#include "klft/klft.hpp"

int main(int argc, char **argv) {
  klft::HMCParams p;
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    const bool has = i + 1 < argc;
    if (a == "--help") {
      std::cout << "Usage: " << argv[0] << " [options]" << std::endl;
      std::cout << "Options:" << std::endl;
      std::cout << "--gauge-group SU2, U1 or SU3" << std::endl;
      std::cout << "--ndim 2, 3, or 4" << std::endl;
      std::cout << "--LX lattice size in x direction" << std::endl;
      std::cout << "--LY lattice size in y direction" << std::endl;
      std::cout << "--LZ lattice size in z direction" << std::endl;
      std::cout << "--LT lattice size in t direction" << std::endl;
      std::cout << "--n-traj number of trajectories" << std::endl;
      std::cout << "--n-steps number of steps in leapfrog" << std::endl;
      std::cout << "--tau trajectory length" << std::endl;
      std::cout << "--beta inverse coupling constant" << std::endl;
      std::cout << "--seed random number generator seed" << std::endl;
      std::cout << "--outfilename output filename" << std::endl;
      std::cout << "--integrator reference (default), leapfrog or omelyan" << std::endl;
      std::cout << "--precision fp64 (default) or mixed" << std::endl;
      std::cout << "--generators reference (default: Pauli / Gell-Mann) or half (t_a/2)" << std::endl;
      std::cout << "-f input file with an HMCParams block" << std::endl;
      return 0;
    }
    if (!has) continue;
    const std::string v = argv[i + 1];
    if (a == "-f" && !klft::parseInputFile(v, p)) return -1;
    if (a == "--gauge-group") p.gauge_group = v;
    if (a == "--ndim") p.ndim = std::stoi(v);
    if (a == "--LX") p.LX = std::stoi(v);
    if (a == "--LY") p.LY = std::stoi(v);
    if (a == "--LZ") p.LZ = std::stoi(v);
    if (a == "--LT") p.LT = std::stoi(v);
    if (a == "--n-traj") p.n_traj = std::stoi(v);
    if (a == "--n-steps") p.n_steps = std::stoi(v);
    if (a == "--tau") p.tau = std::stod(v);
    if (a == "--beta") p.beta = std::stod(v);
    if (a == "--seed") p.seed = std::stoi(v);
    if (a == "--outfilename") p.outfilename = v;
    if (a == "--integrator")
      p.integrator = v == "leapfrog" ? KLFT_INTEGRATOR_LEAPFROG
                     : v == "omelyan" ? KLFT_INTEGRATOR_OMELYAN
                                      : KLFT_INTEGRATOR_REFERENCE_LEAPFROG;
    if (a == "--precision") p.precision = v == "mixed" ? KLFT_PRECISION_MIXED : KLFT_PRECISION_FP64;
    if (a == "--generators") p.generators = v == "half" ? KLFT_GENERATORS_HALF : KLFT_GENERATORS_REFERENCE;
  }
  return klft::HMC(p) == 0 ? 0 : 1;
}
