// Kokkos_Random.hpp -- project-written stand-in for the random pool that klft's
// headers use (Random_XorShift64_Pool).  TEST INFRASTRUCTURE ONLY.
//
// The generator is NOT Kokkos' xorshift: it is the project's counter-based
// Philox4x32-10 stream, so that the reference's own Metropolis functor, run on
// this shim, consumes exactly the random numbers the oracle and the GPU kernels
// consume.  Inside a sublattice launch (a functor exposing `oddeven` and
// `dimensions`) the stream of a thread is keyed on
//   key = (lo32(seed), hi32(seed) ^ chain), ctr = (block, site, step, 1<<24)
// with site = x0 + L0*(x1 + L1*(x2 + L2*x3)) and step = shim::rng_step.
#pragma once
#include "Kokkos_Core.hpp"

namespace Kokkos {
namespace shim {
inline uint32_t rng_step = 0;   // sweep index, set by the harness before each sweep
inline uint64_t rng_chain = 0;

inline void philox(const uint32_t ci[4], const uint32_t ki[2], uint32_t out[4]) {
  uint32_t c0 = ci[0], c1 = ci[1], c2 = ci[2], c3 = ci[3], k0 = ki[0], k1 = ki[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
}  // namespace shim

template <class Space>
class Random_XorShift64 {
 public:
  uint32_t key[2], ctr[4], buf[4];
  int avail = 0;
  bool have_normal = false;
  double spare = 0.0;
  double drand() {
    if (avail == 0) { shim::philox(ctr, key, buf); ctr[0] += 1; avail = 2; }
    uint32_t hi = avail == 2 ? buf[0] : buf[2], lo = avail == 2 ? buf[1] : buf[3];
    avail -= 1;
    return (double)((((uint64_t)hi << 32) | lo) >> 11) * 0x1.0p-53;
  }
  double drand(const double &range) { return range * drand(); }
  double drand(const double &start, const double &end) { return start + drand(end - start); }
  uint64_t urand64() {
    double u = drand();
    return (uint64_t)(u * 0x1.0p53);
  }
  double normal() {
    if (have_normal) { have_normal = false; return spare; }
    double u0 = drand(), u1 = drand();
    double r = std::sqrt(-2.0 * std::log(1.0 - u0)), t = 6.283185307179586 * u1;
    spare = r * std::sin(t);
    have_normal = true;
    return r * std::cos(t);
  }
  double normal(const double &mean, const double &stddev) { return mean + stddev * normal(); }
};

template <class Space>
class Random_XorShift64_Pool {
  uint64_t seed_ = 0;

 public:
  using generator_type = Random_XorShift64<Space>;
  Random_XorShift64_Pool() = default;
  explicit Random_XorShift64_Pool(uint64_t seed) : seed_(seed) {}
  generator_type get_state() const {
    generator_type g;
    g.key[0] = (uint32_t)seed_;
    g.key[1] = (uint32_t)(seed_ >> 32) ^ (uint32_t)shim::rng_chain;
    uint32_t site = 0;
    const auto &c = shim::ctx;
    if (c.active) {
      long s = 0;
      for (int d = c.rank - 1; d >= 0; --d) s = s * (2 * c.half[d]) + (2 * c.idx[d] + c.bits[d]);
      site = (uint32_t)s;
    } else {
      static thread_local uint32_t counter = 0;
      site = (uint32_t)omp_get_thread_num() * 0x10000u + counter++;
    }
    g.ctr[0] = 0; g.ctr[1] = site; g.ctr[2] = shim::rng_step; g.ctr[3] = 1u << 24;
    return g;
  }
  void free_state(const generator_type &) const {}
};

template <class Space> using Random_XorShift1024_Pool = Random_XorShift64_Pool<Space>;

}  // namespace Kokkos
