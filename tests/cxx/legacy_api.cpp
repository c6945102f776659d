// Calls klft's C++ names from include/klft/klft.hpp on one lattice and prints
// the results, one per line, for tests/test_gpu_legacy_api.py:
//   argv: nc L0 L1 L2 L3 seed precision mu nu Lmu Lnu   (L_d = 0: no axis d)
//   out:  plaquette, W normalised, W unnormalised, then the staple field
//         (re im pairs, site-major) as one line of numbers
#include <cstdio>
#include <cstdlib>

#include "klft/klft.hpp"

int main(int argc, char **argv) {
  if (argc != 12) return 2;
  const int nc = atoi(argv[1]);
  int L[4];
  int nd = 0;
  for (int d = 0; d < 4; ++d) {
    L[d] = atoi(argv[2 + d]);
    if (L[d] > 0) nd = d + 1;
  }
  const unsigned long long seed = strtoull(argv[6], nullptr, 10);
  const int precision = atoi(argv[7]);
  const int mu = atoi(argv[8]), nu = atoi(argv[9]), Lmu = atoi(argv[10]), Lnu = atoi(argv[11]);
  for (int d = nd; d < 4; ++d) L[d] = 1;
  klft_lattice *g = nullptr;
  if (klft_lattice_create(nc, nd, L, precision, KLFT_START_HOT, seed, &g) != KLFT_OK) {
    fprintf(stderr, "%s\n", klft_last_error());
    return 1;
  }
  printf("%.17g\n", klft::GaugePlaquette(g));
  printf("%.17g\n", klft::get_W_loop_mu_nu(g, mu, nu, Lmu, Lnu));
  printf("%.17g\n", klft::get_W_loop_mu_nu(g, mu, nu, Lmu, Lnu, false));
  const std::vector<std::complex<double>> st = klft::stapleField(g);
  if (st.empty()) return 1;
  for (const auto &z : st) printf("%.17g %.17g ", z.real(), z.imag());
  printf("\n");
  klft_lattice_destroy(g);
  return 0;
}
