// common.cuh -- device building blocks shared by all kernels of libklft_b200:
// the counter-based random stream, complex and SU(N) matrix algebra templated on
// the storage/arithmetic type T (double: plain FP64 form, float: mixed form),
// and the site geometry of the sublattice-blocked link layout.
//
// Link layout in HBM (structure of arrays, sublattice blocked):
//   element (site x, direction mu, colour entry c = i*Nc + j) lives at
//     links[(mu*Nc*Nc + c) * V + lin(x)]        as a complex of T
//   lin(x) = sub(x) * Vh + hidx(x)
//   sub(x) = sum_d (x_d & 1) << d                (2^Nd parity classes)
//   hidx(x) = h0 + H0*(h1 + H1*(h2 + H2*h3)),  h_d = x_d >> 1,  H_d = L_d / 2
// A parity class is contiguous, so a sublattice pass (the unit of the
// reference's sweep, Metropolis.hpp:139-164) reads its own links and those of
// its neighbours with unit-stride, fully coalesced accesses.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace klft {

#define KLFT_HD __host__ __device__ __forceinline__
#define KLFT_D __device__ __forceinline__

// ------------------------------------------------------------------ random
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
KLFT_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
#else
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

enum StreamKind : uint32_t {
  KIND_METROPOLIS = 1u,  // per (sweep, site): Nd links x nHits hits, in order
  KIND_INIT = 2u,        // per (site, mu): hot-start link
  KIND_MOMENTUM = 3u,    // per (trajectory, site, mu): HMC momenta
  KIND_HMC_ACCEPT = 4u,  // per trajectory: accept/reject uniform
  KIND_SWAP = 5u,        // per (cycle, pair): replica swap uniform
};

// Sequential stream of 53-bit uniforms in [0,1).  key = (lo32(seed),
// hi32(seed) ^ lo32(chain)), counter = (block, site, step, kind<<24 | sub).
// Each Philox block gives two doubles, (w0:w1) then (w2:w3).
struct Stream {
  uint32_t k0, k1, site, step, tag, block;
  uint32_t w[4];
  int avail;
  KLFT_HD Stream(uint64_t seed, uint64_t chain, uint32_t site_, uint32_t step_, uint32_t kind, uint32_t sub)
      : k0((uint32_t)seed), k1((uint32_t)(seed >> 32) ^ (uint32_t)chain), site(site_), step(step_),
        tag((kind << 24) | (sub & 0xFFFFFFu)), block(0), avail(0) {}
  KLFT_HD double next() {
    if (avail == 0) {
      w[0] = block; w[1] = site; w[2] = step; w[3] = tag;
      philox4x32_10(w, k0, k1);
      ++block;
      avail = 2;
    }
    const uint32_t hi = avail == 2 ? w[0] : w[2];
    const uint32_t lo = avail == 2 ? w[1] : w[3];
    --avail;
    return (double)((((uint64_t)hi << 32) | lo) >> 11) * 0x1.0p-53;
  }
  // Kokkos drand(start, end) = start + (end - start) * u
  KLFT_HD double drand(double a, double b) { return a + (b - a) * next(); }
  // Box-Muller pair
  KLFT_D void gauss2(double &g0, double &g1) {
    const double u0 = next(), u1 = next();
    const double r = sqrt(-2.0 * log(1.0 - u0));
    double s, c;
    sincos(6.283185307179586 * u1, &s, &c);
    g0 = r * c;
    g1 = r * s;
  }
};

// ------------------------------------------------------------------ complex
template <typename T> struct cx { T re, im; };

template <typename T> KLFT_HD cx<T> mk(T r, T i) { return cx<T>{r, i}; }
template <typename T> KLFT_HD cx<T> operator+(cx<T> a, cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> KLFT_HD cx<T> operator-(cx<T> a, cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T> KLFT_HD cx<T> operator*(cx<T> a, cx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T> KLFT_HD cx<T> operator*(cx<T> a, T s) { return {a.re * s, a.im * s}; }
template <typename T> KLFT_HD cx<T> operator*(T s, cx<T> a) { return {s * a.re, s * a.im}; }
template <typename T> KLFT_HD cx<T> conj(cx<T> a) { return {a.re, -a.im}; }
template <typename T> KLFT_HD void operator+=(cx<T> &a, cx<T> b) { a.re += b.re; a.im += b.im; }
template <typename T> KLFT_HD void operator-=(cx<T> &a, cx<T> b) { a.re -= b.re; a.im -= b.im; }
// complex / real, as std::complex does it
template <typename T> KLFT_HD cx<T> cdiv(cx<T> a, T s) { return {a.re / s, a.im / s}; }

// ------------------------------------------------------------------ SU(N)
template <int N, typename T> struct Mat { cx<T> e[N][N]; };

template <int N, typename T> KLFT_HD Mat<N, T> mzero() {
  Mat<N, T> m;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) m.e[i][j] = mk<T>(T(0), T(0));
  return m;
}
template <int N, typename T> KLFT_HD Mat<N, T> mident() {
  Mat<N, T> m = mzero<N, T>();
#pragma unroll
  for (int i = 0; i < N; ++i) m.e[i][i] = mk<T>(T(1), T(0));
  return m;
}
// SU(2) elements, and real combinations of them (staple sums, algebra
// elements), have the form [[x, y], [-conj(y), conj(x)]]; so does every product
// of two of them.  The products below form row 0 (in the general order) and
// set row 1 from it: half the multiplications of the general 2x2 product.
template <typename T> KLFT_HD void su2_row1(Mat<2, T> &c) {
  c.e[1][0] = mk<T>(-c.e[0][1].re, c.e[0][1].im);
  c.e[1][1] = mk<T>(c.e[0][0].re, -c.e[0][0].im);
}

// c = a * b (SUN.hpp:28-44 accumulation order)
template <int N, typename T> KLFT_HD Mat<N, T> mul(const Mat<N, T> &a, const Mat<N, T> &b) {
  Mat<N, T> c;
  if constexpr (N == 2) {
    c.e[0][0] = a.e[0][0] * b.e[0][0] + a.e[0][1] * b.e[1][0];
    c.e[0][1] = a.e[0][0] * b.e[0][1] + a.e[0][1] * b.e[1][1];
    su2_row1(c);
    return c;
  }
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      cx<T> s = a.e[i][0] * b.e[0][j];
#pragma unroll
      for (int k = 1; k < N; ++k) s += a.e[i][k] * b.e[k][j];
      c.e[i][j] = s;
    }
  return c;
}
// c = a * b^dagger
template <int N, typename T> KLFT_HD Mat<N, T> mul_nd(const Mat<N, T> &a, const Mat<N, T> &b) {
  Mat<N, T> c;
  if constexpr (N == 2) {
    c.e[0][0] = a.e[0][0] * conj(b.e[0][0]) + a.e[0][1] * conj(b.e[0][1]);
    c.e[0][1] = a.e[0][0] * conj(b.e[1][0]) + a.e[0][1] * conj(b.e[1][1]);
    su2_row1(c);
    return c;
  }
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      cx<T> s = a.e[i][0] * conj(b.e[j][0]);
#pragma unroll
      for (int k = 1; k < N; ++k) s += a.e[i][k] * conj(b.e[j][k]);
      c.e[i][j] = s;
    }
  return c;
}
// c = a^dagger * b^dagger
template <int N, typename T> KLFT_HD Mat<N, T> mul_dd(const Mat<N, T> &a, const Mat<N, T> &b) {
  Mat<N, T> c;
  if constexpr (N == 2) {
    c.e[0][0] = conj(a.e[0][0]) * conj(b.e[0][0]) + conj(a.e[1][0]) * conj(b.e[0][1]);
    c.e[0][1] = conj(a.e[0][0]) * conj(b.e[1][0]) + conj(a.e[1][0]) * conj(b.e[1][1]);
    su2_row1(c);
    return c;
  }
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      cx<T> s = conj(a.e[0][i]) * conj(b.e[j][0]);
#pragma unroll
      for (int k = 1; k < N; ++k) s += conj(a.e[k][i]) * conj(b.e[j][k]);
      c.e[i][j] = s;
    }
  return c;
}
// c = a^dagger * b
template <int N, typename T> KLFT_HD Mat<N, T> mul_dn(const Mat<N, T> &a, const Mat<N, T> &b) {
  Mat<N, T> c;
  if constexpr (N == 2) {
    c.e[0][0] = conj(a.e[0][0]) * b.e[0][0] + conj(a.e[1][0]) * b.e[1][0];
    c.e[0][1] = conj(a.e[0][0]) * b.e[0][1] + conj(a.e[1][0]) * b.e[1][1];
    su2_row1(c);
    return c;
  }
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      cx<T> s = conj(a.e[0][i]) * b.e[0][j];
#pragma unroll
      for (int k = 1; k < N; ++k) s += conj(a.e[k][i]) * b.e[k][j];
      c.e[i][j] = s;
    }
  return c;
}
template <int N, typename T> KLFT_HD Mat<N, T> dagger(const Mat<N, T> &a) {
  Mat<N, T> c;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) c.e[i][j] = conj(a.e[j][i]);
  return c;
}
template <int N, typename T> KLFT_HD void madd(Mat<N, T> &a, const Mat<N, T> &b) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) a.e[i][j] += b.e[i][j];
}
template <int N, typename T> KLFT_HD Mat<N, T> mscale(const Mat<N, T> &a, T s) {
  Mat<N, T> c;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) c.e[i][j] = a.e[i][j] * s;
  return c;
}
// Re Tr(a * b) accumulated over the diagonal as Tr does (SUN.hpp:148-157)
template <int N, typename T> KLFT_HD T retr_mul(const Mat<N, T> &a, const Mat<N, T> &b) {
  T t = T(0);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    cx<T> s = a.e[i][0] * b.e[0][i];
#pragma unroll
    for (int k = 1; k < N; ++k) s += a.e[i][k] * b.e[k][i];
    t += s.re;
  }
  return t;
}
// sum_{ij} Re(a_ij * conj(b_ij)) = Re Tr(a b^dagger)  (GaugePlaquette.hpp:72-79)
template <int N, typename T, typename A> KLFT_HD A retr_nd(const Mat<N, T> &a, const Mat<N, T> &b) {
  A t = A(0);
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) t += (A)a.e[i][j].re * (A)b.e[i][j].re + (A)a.e[i][j].im * (A)b.e[i][j].im;
  return t;
}

// restoreSUN (SUN.hpp:256-340)
template <typename T> KLFT_HD Mat<1, T> restore(const Mat<1, T> &a) {
  Mat<1, T> c;
  const T n = sqrt(a.e[0][0].re * a.e[0][0].re + a.e[0][0].im * a.e[0][0].im);
  if constexpr (sizeof(T) == 4) {
    const T i = T(1) / n;  // FP32: one reciprocal (see the SU(3) form)
    c.e[0][0] = mk<T>(a.e[0][0].re * i, a.e[0][0].im * i);
  } else {
    c.e[0][0] = cdiv(a.e[0][0], n);
  }
  return c;
}
template <typename T> KLFT_HD Mat<2, T> restore(const Mat<2, T> &a) {
  Mat<2, T> c;
  const T n = sqrt(a.e[0][0].re * a.e[0][0].re + a.e[0][0].im * a.e[0][0].im + a.e[0][1].re * a.e[0][1].re +
                   a.e[0][1].im * a.e[0][1].im);
  if constexpr (sizeof(T) == 4) {
    const T r = T(1) / n;  // FP32: one reciprocal (see the SU(3) form)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) c.e[i][j] = mk<T>(a.e[i][j].re * r, a.e[i][j].im * r);
  } else {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) c.e[i][j] = cdiv(a.e[i][j], n);
  }
  return c;
}
template <typename T> KLFT_HD Mat<3, T> restore(const Mat<3, T> &a) {
  Mat<3, T> c;
  const T n0 = sqrt((conj(a.e[0][0]) * a.e[0][0] + conj(a.e[0][1]) * a.e[0][1] + conj(a.e[0][2]) * a.e[0][2]).re);
  const T n1 = sqrt((conj(a.e[1][0]) * a.e[1][0] + conj(a.e[1][1]) * a.e[1][1] + conj(a.e[1][2]) * a.e[1][2]).re);
  if constexpr (sizeof(T) == 4) {
    // FP32: one reciprocal per row (the mixed form has no reference arithmetic
    // to follow; six IEEE divisions per row cost ~3 % of an exp-proposal sweep)
    const T i0 = T(1) / n0, i1 = T(1) / n1;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      c.e[0][j] = mk<T>(a.e[0][j].re * i0, a.e[0][j].im * i0);
      c.e[1][j] = mk<T>(a.e[1][j].re * i1, a.e[1][j].im * i1);
    }
  } else {
#pragma unroll
    for (int j = 0; j < 3; ++j) { c.e[0][j] = cdiv(a.e[0][j], n0); c.e[1][j] = cdiv(a.e[1][j], n1); }
  }
  c.e[2][0] = conj(c.e[0][1] * c.e[1][2] - c.e[0][2] * c.e[1][1]);
  c.e[2][1] = conj(c.e[0][2] * c.e[1][0] - c.e[0][0] * c.e[1][2]);
  c.e[2][2] = conj(c.e[0][0] * c.e[1][1] - c.e[0][1] * c.e[1][0]);
  c.e[1][0] = conj(c.e[2][1] * c.e[0][2] - c.e[2][2] * c.e[0][1]);
  c.e[1][1] = conj(c.e[2][2] * c.e[0][0] - c.e[2][0] * c.e[0][2]);
  c.e[1][2] = conj(c.e[2][0] * c.e[0][1] - c.e[2][1] * c.e[0][0]);
  return c;
}

// ------------------------------------------------------------------ geometry
struct Geom {
  int nd;
  int L[4];      // extents (1 beyond nd)
  int H[4];      // half extents
  int hs[4];     // hidx strides
  long long V, Vh;
  int open_mu;  // open boundary: links U_open_mu on the slice x_open_mu = L - 1 are zero (-1: periodic)
  // select-based access for directions known only at run time, so that a kernel
  // parameter Geom is read from the constant bank instead of a local copy
  KLFT_HD int Ld(int d) const { return d == 0 ? L[0] : (d == 1 ? L[1] : (d == 2 ? L[2] : L[3])); }
  KLFT_HD int Hd(int d) const { return d == 0 ? H[0] : (d == 1 ? H[1] : (d == 2 ? H[2] : H[3])); }
};

// A site as parity bits b_d = x_d & 1 and half-lattice coordinates h_d = x_d / 2.
// Scalar members with select-based access: a direction known only at run time
// (the rolled staple loops) costs a few selects instead of a local-memory array.
struct Site {
  int b0 = 0, b1 = 0, b2 = 0, b3 = 0, h0 = 0, h1 = 0, h2 = 0, h3 = 0;
  KLFT_HD int b(int d) const { return d == 0 ? b0 : (d == 1 ? b1 : (d == 2 ? b2 : b3)); }
  KLFT_HD int h(int d) const { return d == 0 ? h0 : (d == 1 ? h1 : (d == 2 ? h2 : h3)); }
  KLFT_HD void set_b(int d, int v) {
    b0 = d == 0 ? v : b0;
    b1 = d == 1 ? v : b1;
    b2 = d == 2 ? v : b2;
    b3 = d == 3 ? v : b3;
  }
  KLFT_HD void set_h(int d, int v) {
    h0 = d == 0 ? v : h0;
    h1 = d == 1 ? v : h1;
    h2 = d == 2 ? v : h2;
    h3 = d == 3 ? v : h3;
  }
};

KLFT_HD long long site_lin(const Geom &g, const Site &s) {
  int sub = 0;
  long long hidx = 0;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    sub |= s.b(d) << d;
    hidx += (long long)s.h(d) * g.hs[d];
  }
  return (long long)sub * g.Vh + hidx;
}
// a link across the open boundary (zero, never updated)
KLFT_HD bool open_link(const Geom &g, const Site &s, int mu) {
  return mu == g.open_mu && 2 * s.h(mu) + s.b(mu) == g.Ld(mu) - 1;
}
// lexicographic site index, x0 fastest (random-stream key and host layout)
KLFT_HD uint32_t site_lex(const Geom &g, const Site &s) {
  uint32_t lex = 0;
#pragma unroll
  for (int d = 3; d >= 0; --d) lex = lex * (uint32_t)g.L[d] + (uint32_t)(2 * s.h(d) + s.b(d));
  return lex;
}
// x + e_d (periodic)
KLFT_HD Site site_up(const Geom &g, Site s, int d) {
  if (s.b(d) == 0) {
    s.set_b(d, 1);
  } else {
    s.set_b(d, 0);
    s.set_h(d, (s.h(d) + 1 == g.Hd(d)) ? 0 : s.h(d) + 1);
  }
  return s;
}
// x - e_d (periodic)
KLFT_HD Site site_dn(const Geom &g, Site s, int d) {
  if (s.b(d) == 1) {
    s.set_b(d, 0);
  } else {
    s.set_b(d, 1);
    s.set_h(d, (s.h(d) == 0) ? g.Hd(d) - 1 : s.h(d) - 1);
  }
  return s;
}
// x + k e_d, any k >= 0 (periodic)
KLFT_HD Site site_shift(const Geom &g, Site s, int d, int k) {
  int x = 2 * s.h(d) + s.b(d);
  x = (x + k) % g.Ld(d);
  s.set_b(d, x & 1);
  s.set_h(d, x >> 1);
  return s;
}
// Site decodes: 32-bit arithmetic whenever the volume allows (a 64-bit
// division by a run-time extent costs tens of instructions).
KLFT_HD Site site_from_lin(const Geom &g, long long lin) {
  Site s;
  if (g.V < (1LL << 31)) {
    const unsigned vh = (unsigned)g.Vh, sub = (unsigned)lin / vh;
    unsigned hidx = (unsigned)lin - sub * vh;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      const unsigned hd = (unsigned)g.H[d], q = hidx / hd;
      s.set_b(d, (int)((sub >> d) & 1u));
      s.set_h(d, (int)(hidx - q * hd));
      hidx = q;
    }
    return s;
  }
  const int sub = (int)(lin / g.Vh);
  long long hidx = lin - (long long)sub * g.Vh;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    s.set_b(d, (sub >> d) & 1);
    s.set_h(d, (int)(hidx % g.H[d]));
    hidx /= g.H[d];
  }
  return s;
}
KLFT_HD Site site_from_lex(const Geom &g, long long lex) {
  Site s;
  if (g.V < (1LL << 31)) {
    unsigned r = (unsigned)lex;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      const unsigned ld = (unsigned)g.L[d], q = r / ld;
      const int x = (int)(r - q * ld);
      r = q;
      s.set_b(d, x & 1);
      s.set_h(d, x >> 1);
    }
    return s;
  }
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const int x = (int)(lex % g.L[d]);
    lex /= g.L[d];
    s.set_b(d, x & 1);
    s.set_h(d, x >> 1);
  }
  return s;
}

// ------------------------------------------------------------------ link field view
// Stored colour planes per link: all N*N, except in the mixed (FP32) form
// SU(3), which keeps rows 0 and 1 (12 reals) and rebuilds row 2 as
// conj(row0 x row1), the unit-determinant completion of two orthonormal rows,
// and SU(2), which keeps row 0 (a, b) (4 reals) and rebuilds row 1 as
// (-conj(b), conj(a)).
template <int N, typename T> struct LinkPlanes { static constexpr int n = N * N; };
template <> struct LinkPlanes<3, float> { static constexpr int n = 6; };
template <> struct LinkPlanes<2, float> { static constexpr int n = 2; };
KLFT_HD int link_planes(int nc, int dtype) {
  return dtype == 1 && nc == 3 ? 6 : (dtype == 1 && nc == 2 ? 2 : nc * nc);
}

template <int N, typename T> struct Links {
  cx<T> *p;
  long long V;
  static constexpr int P = LinkPlanes<N, T>::n;
  KLFT_D Mat<N, T> load(long long lin, int mu) const {
    Mat<N, T> m;
    const cx<T> *q = p + (long long)mu * P * V + lin;
    if constexpr (P == N * N) {
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) m.e[i][j] = q[(i * N + j) * V];
    } else if constexpr (N == 3) {
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) m.e[i][j] = q[(i * 3 + j) * V];
      m.e[2][0] = conj(m.e[0][1] * m.e[1][2] - m.e[0][2] * m.e[1][1]);
      m.e[2][1] = conj(m.e[0][2] * m.e[1][0] - m.e[0][0] * m.e[1][2]);
      m.e[2][2] = conj(m.e[0][0] * m.e[1][1] - m.e[0][1] * m.e[1][0]);
    } else {
      m.e[0][0] = q[0];
      m.e[0][1] = q[V];
      m.e[1][0] = mk<T>(-m.e[0][1].re, m.e[0][1].im);
      m.e[1][1] = conj(m.e[0][0]);
    }
    return m;
  }
  // rows 0 and 1 only (row 2 left unset), for callers that never read it
  KLFT_D Mat<N, T> load_rows01(long long lin, int mu) const {
    Mat<N, T> m;
    const cx<T> *q = p + (long long)mu * P * V + lin;
#pragma unroll
    for (int i = 0; i < (N < 2 ? N : 2); ++i)
#pragma unroll
      for (int j = 0; j < N; ++j) m.e[i][j] = q[(i * N + j) * V];
    return m;
  }
  KLFT_D void store(long long lin, int mu, const Mat<N, T> &m) const {
    cx<T> *q = p + (long long)mu * P * V + lin;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int j = 0; j < N; ++j)
        if ((i * N + j) < P) q[(i * N + j) * V] = m.e[i][j];
  }
};

// PTBC boundary defect (PTBCGaugeField.hpp:30-36, :187-198): links mu = 0 at
// x0 = 0 whose x_1..x_{Nd-1} lie in pos + [0, len) (periodic) carry factor c.
struct Defect {
  int active;
  int len;
  int pos[3];
  double c;
  const double *dyn_c;  // when set, the factor is read from device memory (replica swaps inside a graph)
};
KLFT_HD double defect_c(const Defect &df) {
#ifdef __CUDA_ARCH__
  return df.dyn_c ? *df.dyn_c : df.c;
#else
  return df.c;
#endif
}
KLFT_HD bool in_defect(const Geom &g, const Defect &df, const Site &s, int mu) {
  if (!df.active || mu != 0) return false;
  if (2 * s.h(0) + s.b(0) != 0) return false;
  for (int d = 1; d < g.nd; ++d) {
    int rel = (2 * s.h(d) + s.b(d)) - df.pos[d - 1];
    rel %= g.L[d];
    if (rel < 0) rel += g.L[d];
    if (rel >= df.len) return false;
  }
  return true;
}

// ------------------------------------------------------------------ reductions
template <typename A> KLFT_D A warp_sum(A v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace klft
