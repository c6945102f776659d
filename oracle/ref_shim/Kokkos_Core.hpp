// Kokkos_Core.hpp -- project-written host shim of the small part of the Kokkos
// API that klft's headers use, so that the reference's own headers compile
// unchanged on the CPU (OpenMP).  TEST INFRASTRUCTURE ONLY (oracle/_ref).
//
// Written from the public Kokkos API documentation (View, Array, complex,
// MDRangePolicy, parallel_for/parallel_reduce, fence, Timer).  It is not the
// Kokkos OpenMP backend: views are LayoutRight host arrays, MDRange loops are
// OpenMP loops over the two outermost indices.
#pragma once

#include <algorithm>
#include <cassert>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

#include <omp.h>

#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [ =, *this ]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_ENABLE_OPENMP 1

// klft/include/GaugeField.hpp names `site` in three openBC() bodies where no
// such variable is in scope.  The bodies are never instantiated; g++ only needs
// the name to resolve at template definition time.
inline int site = 0;

namespace Kokkos {

// ------------------------------------------------------------------ basics
struct OpenMP {};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

inline void initialize() {}
inline void initialize(int &, char **) {}
inline void finalize() {}
inline void fence() {}

namespace numbers {
template <class T> inline constexpr T pi_v = T(3.141592653589793238462643383279502884L);
}

template <class T> using complex = std::complex<T>;
using std::conj;
using std::cos;
using std::exp;
using std::real;
using std::sin;
using std::sqrt;

class Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

 public:
  void reset() { t0 = std::chrono::steady_clock::now(); }
  double seconds() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

// ------------------------------------------------------------------ Array
template <class T, size_t N>
struct Array {
  T m[N > 0 ? N : 1];
  Array() = default;
  template <class... Ts, class = std::enable_if_t<(sizeof...(Ts) > 0) && (sizeof...(Ts) <= N) &&
                                                  (std::is_convertible_v<Ts, T> && ...)>>
  Array(Ts... ts) : m{static_cast<T>(ts)...} {}
  template <class U, class = std::enable_if_t<!std::is_same_v<U, T> && std::is_convertible_v<U, T>>>
  Array(const Array<U, N> &o) {
    for (size_t i = 0; i < N; ++i) m[i] = static_cast<T>(o.m[i]);
  }
  T &operator[](size_t i) { return m[i]; }
  const T &operator[](size_t i) const { return m[i]; }
  static constexpr size_t size() { return N; }
  T *data() { return m; }
  const T *data() const { return m; }
  T *begin() { return m; }
  T *end() { return m + N; }
  const T *begin() const { return m; }
  const T *end() const { return m + N; }
};

// ------------------------------------------------------------------ View
struct WithoutInitializing_t {};
inline constexpr WithoutInitializing_t WithoutInitializing{};
struct Restrict {};
struct RandomAccess {};
template <class... > struct MemoryTraits {};
struct LayoutRight {
  size_t dimension[8];
};

namespace detail {
template <class T> struct vparse {
  using value_type = T;
  static constexpr int ndyn = 0;
  static constexpr int nstat = 0;
  static constexpr size_t stat = 1;
};
template <class T> struct vparse<T *> {
  using value_type = typename vparse<T>::value_type;
  static constexpr int ndyn = vparse<T>::ndyn + 1;
  static constexpr int nstat = vparse<T>::nstat;
  static constexpr size_t stat = vparse<T>::stat;
};
template <class T, size_t N> struct vparse<T[N]> {
  using value_type = typename vparse<T>::value_type;
  static constexpr int ndyn = vparse<T>::ndyn;
  static constexpr int nstat = vparse<T>::nstat + 1;
  static constexpr size_t stat = N;
};
}  // namespace detail

template <class DataType, class... Props>
class View {
  using P = detail::vparse<DataType>;

 public:
  using value_type = typename P::value_type;
  using nc_value_type = std::remove_const_t<value_type>;
  static constexpr int rank_dynamic = P::ndyn;
  static constexpr int rank = P::ndyn + P::nstat;

  std::shared_ptr<nc_value_type> store;
  value_type *ptr = nullptr;
  size_t ext[8] = {0, 0, 0, 0, 0, 0, 0, 0};

  View() = default;
  template <class... Is>
  explicit View(const std::string &, Is... dims) {
    alloc(size_t(dims)...);
  }
  template <class D2, class... P2>
  View(const View<D2, P2...> &o) : store(o.store), ptr(o.ptr) {
    for (int i = 0; i < 8; ++i) ext[i] = o.ext[i];
  }

  template <class... Is>
  void alloc(Is... dims) {
    static_assert(sizeof...(Is) == rank_dynamic, "dynamic extents");
    size_t d[] = {size_t(dims)...};
    size_t n = 1;
    for (int i = 0; i < rank_dynamic; ++i) { ext[i] = d[i]; n *= d[i]; }
    if (P::nstat) { ext[rank_dynamic] = P::stat; n *= P::stat; }
    for (int i = rank; i < 8; ++i) ext[i] = 1;
    store = std::shared_ptr<nc_value_type>(new nc_value_type[n > 0 ? n : 1](), std::default_delete<nc_value_type[]>());
    ptr = store.get();
  }

  size_t span() const {
    size_t n = 1;
    for (int i = 0; i < rank; ++i) n *= ext[i];
    return n;
  }
  size_t extent(int i) const { return ext[i]; }
  LayoutRight layout() const {
    LayoutRight l;
    for (int i = 0; i < 8; ++i) l.dimension[i] = ext[i];
    return l;
  }
  value_type *data() const { return ptr; }

  template <class... Is>
  value_type &operator()(Is... is) const {
    static_assert(sizeof...(Is) == rank, "view rank");
    size_t idx[] = {size_t(is)...};
    size_t off = 0;
    for (int i = 0; i < rank; ++i) off = off * ext[i] + idx[i];
    return ptr[off];
  }
};

template <class D, class... P, class... Is>
void realloc(WithoutInitializing_t, View<D, P...> &v, Is... dims) {
  v.alloc(dims...);
}
template <class D, class... P, class... Is>
void realloc(View<D, P...> &v, Is... dims) {
  v.alloc(dims...);
}

template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...> &dst, const View<D2, P2...> &src) {
  const size_t n = std::min(dst.span(), src.span());
  for (size_t i = 0; i < n; ++i) dst.ptr[i] = src.ptr[i];
}

// ------------------------------------------------------------------ policies
template <unsigned R> struct Rank { static constexpr unsigned rank = R; };

template <class RankT>
struct MDRangePolicy {
  static constexpr int R = RankT::rank;
  Array<long, R> lo, hi, tile;
  MDRangePolicy(const Array<long, R> &s, const Array<long, R> &e) : lo(s), hi(e) {
    for (int i = 0; i < R; ++i) tile[i] = 1;
  }
  template <class A, class B>
  MDRangePolicy(const A &s, const B &e) {
    for (int i = 0; i < R; ++i) { lo[i] = s[i]; hi[i] = e[i]; tile[i] = 1; }
  }
  template <class A, class B, class C>
  MDRangePolicy(const A &s, const B &e, const C &t) {
    for (int i = 0; i < R; ++i) { lo[i] = s[i]; hi[i] = e[i]; tile[i] = t[i]; }
  }
  long max_total_tile_size() const { return 1024; }
};

template <class... > struct RangePolicy {
  long lo = 0, hi = 0;
  RangePolicy(long e) : hi(e) {}
  RangePolicy(long s, long e) : lo(s), hi(e) {}
};

// Hook for the harness: runs before each MDRange iteration so that a random
// pool can key its stream on the iteration.  Set by Kokkos_Random.hpp users.
namespace shim {
template <class F, class = void> struct has_oddeven : std::false_type {};
template <class F>
struct has_oddeven<F, std::void_t<decltype(std::declval<const F &>().oddeven),
                                  decltype(std::declval<const F &>().dimensions)>> : std::true_type {};

struct IterCtx {
  int active = 0;        // 1 inside a sublattice (Metropolis) launch
  int rank = 0;
  int bits[8] = {0};     // sublattice parity per dimension
  long half[8] = {0};    // half extents
  long idx[8] = {0};     // current iteration index
};
inline thread_local IterCtx ctx;
}  // namespace shim

template <int R, class F, class Red = void>
inline void md_loop(const MDRangePolicy<Rank<R>> &p, const F &f) {
  constexpr bool keyed = shim::has_oddeven<F>::value;
  if constexpr (R == 1) {
#pragma omp parallel for schedule(static)
    for (long i0 = p.lo[0]; i0 < p.hi[0]; ++i0) f((int)i0);
  } else {
    const long n0 = p.hi[0] - p.lo[0], n1 = p.hi[1] - p.lo[1];
#pragma omp parallel for collapse(2) schedule(static)
    for (long a = 0; a < n0; ++a)
      for (long b = 0; b < n1; ++b) {
        const int i0 = (int)(p.lo[0] + a), i1 = (int)(p.lo[1] + b);
        if constexpr (keyed) {
          shim::ctx.active = 1;
          shim::ctx.rank = R;
          for (int d = 0; d < R; ++d) { shim::ctx.bits[d] = f.oddeven[d] ? 1 : 0; shim::ctx.half[d] = f.dimensions[d]; }
          shim::ctx.idx[0] = i0;
          shim::ctx.idx[1] = i1;
        }
        if constexpr (R == 2) {
          f(i0, i1);
        } else if constexpr (R == 3) {
          for (long i2 = p.lo[2]; i2 < p.hi[2]; ++i2) {
            if constexpr (keyed) shim::ctx.idx[2] = i2;
            f(i0, i1, (int)i2);
          }
        } else if constexpr (R == 4) {
          for (long i2 = p.lo[2]; i2 < p.hi[2]; ++i2)
            for (long i3 = p.lo[3]; i3 < p.hi[3]; ++i3) {
              if constexpr (keyed) { shim::ctx.idx[2] = i2; shim::ctx.idx[3] = i3; }
              f(i0, i1, (int)i2, (int)i3);
            }
        } else if constexpr (R == 5) {
          for (long i2 = p.lo[2]; i2 < p.hi[2]; ++i2)
            for (long i3 = p.lo[3]; i3 < p.hi[3]; ++i3)
              for (long i4 = p.lo[4]; i4 < p.hi[4]; ++i4) f(i0, i1, (int)i2, (int)i3, (int)i4);
        }
        if constexpr (keyed) shim::ctx.active = 0;
      }
  }
}

template <unsigned R, class F>
inline void parallel_for(const MDRangePolicy<Rank<R>> &p, const F &f) {
  md_loop<(int)R>(p, f);
}
template <unsigned R, class F>
inline void parallel_for(const std::string &, const MDRangePolicy<Rank<R>> &p, const F &f) {
  md_loop<(int)R>(p, f);
}
template <class... X, class F>
inline void parallel_for(const RangePolicy<X...> &p, const F &f) {
#pragma omp parallel for schedule(static)
  for (long i = p.lo; i < p.hi; ++i) f((int)i);
}
template <class... X, class F>
inline void parallel_for(const std::string &, const RangePolicy<X...> &p, const F &f) {
  parallel_for(p, f);
}

template <class T> struct Sum {
  T &ref;
  explicit Sum(T &r) : ref(r) {}
};

// Deterministic for a fixed thread count: per-thread partial sums over a
// static schedule, combined in thread order.
template <unsigned R, class F, class T>
inline void parallel_reduce(const std::string &, const MDRangePolicy<Rank<R>> &p, const F &f, Sum<T> red) {
  const int nt = omp_get_max_threads();
  std::vector<T> part((size_t)nt, T());
  const long n0 = p.hi[0] - p.lo[0];
#pragma omp parallel num_threads(nt)
  {
    T loc = T();
    const int tid = omp_get_thread_num();
#pragma omp for schedule(static)
    for (long a = 0; a < n0; ++a) {
      const int i0 = (int)(p.lo[0] + a);
      if constexpr (R == 2) {
        for (long i1 = p.lo[1]; i1 < p.hi[1]; ++i1) f(i0, (int)i1, loc);
      } else if constexpr (R == 3) {
        for (long i1 = p.lo[1]; i1 < p.hi[1]; ++i1)
          for (long i2 = p.lo[2]; i2 < p.hi[2]; ++i2) f(i0, (int)i1, (int)i2, loc);
      } else if constexpr (R == 4) {
        for (long i1 = p.lo[1]; i1 < p.hi[1]; ++i1)
          for (long i2 = p.lo[2]; i2 < p.hi[2]; ++i2)
            for (long i3 = p.lo[3]; i3 < p.hi[3]; ++i3) f(i0, (int)i1, (int)i2, (int)i3, loc);
      }
    }
    part[(size_t)tid] = loc;
  }
  T total = T();
  for (const T &x : part) total += x;
  red.ref = total;
}

}  // namespace Kokkos
