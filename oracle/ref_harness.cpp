// ref_harness.cpp -- drives klft's own headers (compiled unchanged from the
// reference tree, -I<reference>/include) on the CPU through the project's
// Kokkos-API shim in ref_shim/.  TEST INFRASTRUCTURE ONLY: used by tests/ to
// pin the oracle and by bench.py's reference arm / cpu_baseline leg.
//
// Host arrays use the interchange layout of oracle.cpp:
//   U[(((site*Nd + mu)*Nc + i)*Nc + j)] complex<double>, site = x0 + L0*(x1 + ...).
#include <Kokkos_Core.hpp>
#include <Kokkos_Random.hpp>

#include "Metropolis.hpp"   // klft: sweep_Metropolis, run_metropolis, observables
#include "Gauge_Util.hpp"   // klft: stapleField (4D)

using namespace klft;
using cplx = std::complex<double>;

namespace {

template <size_t rank, size_t Nc>
typename DeviceGaugeFieldType<rank, Nc>::type make_field(const int *L) {
  if constexpr (rank == 4) return deviceGaugeField<4, Nc>(L[0], L[1], L[2], L[3], identitySUN<Nc>());
  else if constexpr (rank == 3) return deviceGaugeField3D<3, Nc>(L[0], L[1], L[2], identitySUN<Nc>());
  else return deviceGaugeField2D<2, Nc>(L[0], L[1], identitySUN<Nc>());
}

template <size_t rank>
long lex(const int *x, const int *L) {
  long s = 0;
  for (int d = (int)rank - 1; d >= 0; --d) s = s * L[d] + x[d];
  return s;
}

template <size_t rank, size_t Nc, class G, class Fn>
void for_links(const G &g, const int *L, Fn fn) {
  int x[4] = {0, 0, 0, 0};
  long V = 1;
  for (size_t d = 0; d < rank; ++d) V *= L[d];
  for (long s = 0; s < V; ++s) {
    long t = s;
    for (size_t d = 0; d < rank; ++d) { x[d] = (int)(t % L[d]); t /= L[d]; }
    for (size_t mu = 0; mu < rank; ++mu) {
      SUN<Nc> *p;
      if constexpr (rank == 4) p = &g.field(x[0], x[1], x[2], x[3], mu);
      else if constexpr (rank == 3) p = &g.field(x[0], x[1], x[2], mu);
      else p = &g.field(x[0], x[1], mu);
      fn(*p, (s * (long)rank + (long)mu) * (long)(Nc * Nc));
    }
  }
}

template <size_t rank, size_t Nc, class G>
void load(G &g, const int *L, const double *U) {
  const cplx *u = (const cplx *)U;
  for_links<rank, Nc>(g, L, [&](SUN<Nc> &m, long off) {
    for (size_t i = 0; i < Nc; ++i) for (size_t j = 0; j < Nc; ++j) m[i][j] = u[off + i * Nc + j];
  });
}
template <size_t rank, size_t Nc, class G>
void store(const G &g, const int *L, double *U) {
  cplx *u = (cplx *)U;
  for_links<rank, Nc>(g, L, [&](SUN<Nc> &m, long off) {
    for (size_t i = 0; i < Nc; ++i) for (size_t j = 0; j < Nc; ++j) u[off + i * Nc + j] = m[i][j];
  });
}

std::vector<Kokkos::Array<index_t, 2>> to_pairs(const int *pairs, int n) {
  std::vector<Kokkos::Array<index_t, 2>> v;
  for (int k = 0; k < n; ++k) v.push_back({pairs[2 * k], pairs[2 * k + 1]});
  return v;
}

template <size_t rank, size_t Nc>
void set_params(MetropolisParams &p, const int *L, double beta, double delta, int nHits, int seed) {
  p.Ndims = (index_t)rank;
  p.Nd = rank;
  p.Nc = Nc;
  p.L0 = L[0]; p.L1 = L[1];
  p.L2 = rank > 2 ? L[2] : 1;
  p.L3 = rank > 3 ? L[3] : 1;
  p.nHits = nHits;
  p.beta = beta;
  p.delta = delta;
  p.seed = seed;
}

}  // namespace

#define DISPATCH(nd, nc, BODY)                                                        \
  do {                                                                                \
    if (nd == 4 && nc == 1) { constexpr size_t R = 4, N = 1; BODY; }                  \
    else if (nd == 4 && nc == 2) { constexpr size_t R = 4, N = 2; BODY; }             \
    else if (nd == 4 && nc == 3) { constexpr size_t R = 4, N = 3; BODY; }             \
    else if (nd == 3 && nc == 1) { constexpr size_t R = 3, N = 1; BODY; }             \
    else if (nd == 3 && nc == 2) { constexpr size_t R = 3, N = 2; BODY; }             \
    else if (nd == 3 && nc == 3) { constexpr size_t R = 3, N = 3; BODY; }             \
    else if (nd == 2 && nc == 1) { constexpr size_t R = 2, N = 1; BODY; }             \
    else if (nd == 2 && nc == 2) { constexpr size_t R = 2, N = 2; BODY; }             \
    else if (nd == 2 && nc == 3) { constexpr size_t R = 2, N = 3; BODY; }             \
    else return -1;                                                                   \
  } while (0)

extern "C" {

int ref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// GaugePlaquette.hpp:89-135
int ref_plaquette(int nc, int nd, const int *L, const double *U, double *out) {
  DISPATCH(nd, nc, ({
    auto g = make_field<R, N>(L);
    load<R, N>(g, L, U);
    *out = GaugePlaquette<R, N>(g);
  }));
  return 0;
}

// WilsonLoop.hpp:250-304
int ref_wilson_temporal(int nc, int nd, const int *L, const double *U, const int *pairs, int n, double *out) {
  DISPATCH(nd, nc, ({
    auto g = make_field<R, N>(L);
    load<R, N>(g, L, U);
    std::vector<Kokkos::Array<real_t, 3>> vals;
    WilsonLoop_temporal<R, N>(g, to_pairs(pairs, n), vals);
    for (int k = 0; k < n; ++k) out[k] = vals[k][2];
  }));
  return 0;
}

// WilsonLoop.hpp:170-245
int ref_wilson_mu_nu(int nc, int nd, const int *L, const double *U, int mu, int nu, const int *pairs, int n,
                     double *out) {
  DISPATCH(nd, nc, ({
    auto g = make_field<R, N>(L);
    load<R, N>(g, L, U);
    std::vector<Kokkos::Array<real_t, 5>> vals;
    WilsonLoop_mu_nu<R, N>(g, mu, nu, to_pairs(pairs, n), vals);
    for (int k = 0; k < n; ++k) out[k] = vals[k][4];
  }));
  return 0;
}

// Gauge_Util.hpp:27-97 (4D only)
int ref_staple_field(int nc, const int *L, const double *U, double *out) {
  DISPATCH(4, nc, ({
    if constexpr (R == 4) {
      auto g = make_field<4, N>(L);
      load<4, N>(g, L, U);
      auto st = stapleField<4, N>(g);
      cplx *o = (cplx *)out;
      const long V = (long)L[0] * L[1] * L[2] * L[3];
      int x[4];
      for (long s = 0; s < V; ++s) {
        long t = s;
        for (int d = 0; d < 4; ++d) { x[d] = (int)(t % L[d]); t /= L[d]; }
        for (int mu = 0; mu < 4; ++mu) {
          const SUN<N> &m = st(x[0], x[1], x[2], x[3], mu);
          for (size_t i = 0; i < N; ++i)
            for (size_t j = 0; j < N; ++j) o[((s * 4 + mu) * (long)N + (long)i) * (long)N + (long)j] = m[i][j];
        }
      }
    }
  }));
  return 0;
}

// Metropolis.hpp:118-178, one call per sweep; shim::rng_step carries the sweep index
int ref_metropolis(int nc, int nd, const int *L, double *U, double beta, double delta, int nHits, int seed,
                   uint32_t sweep0, int nsweeps, double *acc_out) {
  DISPATCH(nd, nc, ({
    auto g = make_field<R, N>(L);
    load<R, N>(g, L, U);
    MetropolisParams p;
    set_params<R, N>(p, L, beta, delta, nHits, seed);
    RNGType rng(seed);
    for (int k = 0; k < nsweeps; ++k) {
      Kokkos::shim::rng_step = sweep0 + (uint32_t)k;
      acc_out[k] = sweep_Metropolis<R, N>(g, p, rng);
    }
    store<R, N>(g, L, U);
  }));
  return 0;
}

// One update-and-measure cycle as run_metropolis does it (Metropolis.hpp:204-218):
// a sweep, then GaugePlaquette and WilsonLoop_temporal.  Used as the timed CPU
// baseline.  U is loaded once per call; nsweeps cycles run back to back.
int ref_cycles(int nc, int nd, const int *L, double *U, double beta, double delta, int nHits, int seed,
               uint32_t sweep0, int nsweeps, const int *pairs, int npairs, double *acc_out, double *plaq_out,
               double *w_out) {
  DISPATCH(nd, nc, ({
    auto g = make_field<R, N>(L);
    load<R, N>(g, L, U);
    MetropolisParams p;
    set_params<R, N>(p, L, beta, delta, nHits, seed);
    RNGType rng(seed);
    auto pv = to_pairs(pairs, npairs);
    for (int k = 0; k < nsweeps; ++k) {
      Kokkos::shim::rng_step = sweep0 + (uint32_t)k;
      acc_out[k] = sweep_Metropolis<R, N>(g, p, rng);
      plaq_out[k] = GaugePlaquette<R, N>(g);
      if (npairs > 0) {
        std::vector<Kokkos::Array<real_t, 3>> vals;
        WilsonLoop_temporal<R, N>(g, pv, vals);
        for (int q = 0; q < npairs; ++q) w_out[(long)k * npairs + q] = vals[q][2];
      }
    }
    store<R, N>(g, L, U);
  }));
  return 0;
}

}  // extern "C"
