// wilson.cu -- Wilson loops in a (mu, nu) plane by axial gauge fixing.
//
// Reference semantics (WilsonLoop.hpp:101-245): for each requested (Lmu, Lnu)
//   W = Re sum_x Tr[ WLmu(x) WLnu(x + Lmu mu) (WLnu(x) WLmu(x + Lnu nu))^+ ]
// with WL_d(x) the product of links along d.  Loops are gauge invariant, so
// each (mu, nu) plane may be computed in its own gauge.  With
//   Omega(x) = U_nu(xbar,0) U_nu(xbar,1) ... U_nu(xbar, x_nu - 1)   (Omega = 1 at x_nu = 0)
// the transformed links U'_nu are the identity except on the last row, and
//   U'_mu(x) = Omega(x) U_mu(x) Omega(x + mu)^+.
// The spatial line S'_L(x) = U'_mu(x) ... U'_mu(x + (L-1) mu) then gives
//   W_{L,T}(x) = Re Tr[ S'_L(x) S'_L(x + T nu)^+ ]
// once rows past the end of the nu axis are continued with the Polyakov line
// P(xbar) = Omega(xbar, L_nu):  U'_mu(xbar, b + k L_nu) = P^k U'_mu(xbar, b) P(xbar + mu)^-k.
// Per (site, L, T) the loop costs one trace of a product (18 FMAs for SU(3))
// instead of the ~4 matrix products of the direct form.
//
// Kernels: omega_kernel (per nu: the axial-gauge transformation, products in
// FP64, stored in the link precision), uprime_kernel (per plane: U'_mu on
// L_nu + T_max rows in the link precision), wcorr_kernel (the column-correlation
// form below, all planes of one nu in one launch), wloop_kernel (per plane: persistent CTAs over
// tiles of CW columns x R rows; S'_L is built incrementally over L in shared
// memory together with a halo of T_max rows of the same column; per-site traces
// in the link precision, lattice sums in FP64).
//
// Omega is stored row major (row b, column c at b*ncols + c) and U' column major
// (c*rows + b), one plane per complex colour entry: the kernels that write them
// run lanes over columns, the loop kernel reads U' with lanes over rows.
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"

namespace klft {

struct ColGeom {
  int nd, mu, nu;
  int L[4];
  int cs[4];      // column stride of each dimension (0 for nu)
  long long ncols;
  int rows;       // stored rows of U' (L_nu + extension)
  int Lmu, Lnu, csmu;  // L[mu], L[nu], cs[mu] (kernel parameters indexed by a run-time mu would be copied)
};

KLFT_HD ColGeom make_colgeom(const Geom &g, int mu, int nu, int rows) {
  ColGeom c;
  c.nd = g.nd;
  c.mu = mu;
  c.nu = nu;
  long long s = 1;
  for (int d = 0; d < 4; ++d) {
    c.L[d] = g.L[d];
    if (d == nu || d >= g.nd) {
      c.cs[d] = 0;
    } else {
      c.cs[d] = (int)s;
      s *= g.L[d];
    }
  }
  c.ncols = s;
  c.rows = rows;
  c.Lmu = g.L[mu];
  c.Lnu = g.L[nu];
  c.csmu = c.cs[mu];
  return c;
}

// Coordinates of a column along the dimensions other than nu (x[nu] = 0), in
// 32-bit arithmetic whenever the column count allows it (a 64-bit division
// by a run-time extent costs several times a 3x3 product).
KLFT_D void col_coords(const ColGeom &c, long long col, int x[4]) {
  if (c.ncols <= 0xffffffffLL) {
    unsigned u = (unsigned)col;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      if (d == c.nu || d >= c.nd) {
        x[d] = 0;
      } else {
        const unsigned Ld = (unsigned)c.L[d], qd = u / Ld;
        x[d] = (int)(u - qd * Ld);
        u = qd;
      }
    }
  } else {
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      if (d == c.nu || d >= c.nd) {
        x[d] = 0;
      } else {
        x[d] = (int)(col % c.L[d]);
        col /= c.L[d];
      }
    }
  }
}

// site of the column with coordinates x at row < L_nu
KLFT_D Site col_site_at(const ColGeom &c, const int x[4], int row) {
  Site s;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const int v = d == c.nu ? row : x[d];
    s.set_b(d, v & 1);
    s.set_h(d, v >> 1);
  }
  return s;
}

// column index of xbar + k mu, with xm the column's coordinate along mu
KLFT_D long long col_shift_at(const ColGeom &c, long long col, int xm, int k) {
  const int xn = (xm + k) % c.Lmu;
  return col + (long long)(xn - xm) * c.csmu;
}

// Scratch field of N x N complex entries per site.  FP64: one plane per entry
// (entry a of site i at a * n + i, 16 bytes).  FP32: entries in pairs, so that
// a thread moves 16 bytes per access: entries 2q and 2q + 1 of site i share the
// 16-byte slot q * n + i (CPairs<N> pair planes; an odd last entry has its slot
// to itself).
template <int N> struct CPairs { static constexpr int v = (N * N + 1) / 2; };
template <int N, typename T> struct CField {
  cx<T> *p;
  long long n;  // sites per plane
  static constexpr bool paired = sizeof(T) == 4;
  KLFT_D cx<T> get(int a, long long i) const {
    if constexpr (paired) return p[((long long)(a >> 1) * n + i) * 2 + (a & 1)];
    else return p[(long long)a * n + i];
  }
  KLFT_D Mat<N, T> load_t(long long i) const {
    Mat<N, T> m;
    if constexpr (paired) {
#pragma unroll
      for (int q = 0; q < CPairs<N>::v; ++q) {
        const float4 v = ((const float4 *)p)[(long long)q * n + i];
        m.e[(2 * q) / N][(2 * q) % N] = mk<T>(v.x, v.y);
        if (2 * q + 1 < N * N) m.e[(2 * q + 1) / N][(2 * q + 1) % N] = mk<T>(v.z, v.w);
      }
    } else {
#pragma unroll
      for (int a = 0; a < N; ++a)
#pragma unroll
        for (int b = 0; b < N; ++b) m.e[a][b] = p[(a * N + b) * n + i];
    }
    return m;
  }
  KLFT_D Mat<N, double> load(long long i) const {
    const Mat<N, T> t = load_t(i);
    Mat<N, double> m;
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int b = 0; b < N; ++b) m.e[a][b] = mk<double>((double)t.e[a][b].re, (double)t.e[a][b].im);
    return m;
  }
  KLFT_D void store_t(long long i, const Mat<N, T> &m) const {
    if constexpr (paired) {
#pragma unroll
      for (int q = 0; q < CPairs<N>::v; ++q) {
        const cx<T> x = m.e[(2 * q) / N][(2 * q) % N];
        const cx<T> y = 2 * q + 1 < N * N ? m.e[(2 * q + 1) / N][(2 * q + 1) % N] : mk<T>(T(0), T(0));
        ((float4 *)p)[(long long)q * n + i] = make_float4(x.re, x.im, y.re, y.im);
      }
    } else {
#pragma unroll
      for (int a = 0; a < N; ++a)
#pragma unroll
        for (int b = 0; b < N; ++b) p[(a * N + b) * n + i] = m.e[a][b];
    }
  }
  KLFT_D void store(long long i, const Mat<N, double> &m) const {
    Mat<N, T> t;
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int b = 0; b < N; ++b) t.e[a][b] = mk<T>((T)m.e[a][b].re, (T)m.e[a][b].im);
    store_t(i, t);
  }
  // bytes of one field of nsites sites
  static KLFT_HD size_t bytes(long long nsites) {
    return (size_t)nsites * (paired ? 2 * CPairs<N>::v : N * N) * sizeof(cx<T>);
  }
};

template <int N, typename T> KLFT_D Mat<N, double> to_d(const Mat<N, T> &m) {
  Mat<N, double> r;
#pragma unroll
  for (int a = 0; a < N; ++a)
#pragma unroll
    for (int b = 0; b < N; ++b) r.e[a][b] = mk<double>((double)m.e[a][b].re, (double)m.e[a][b].im);
  return r;
}

// Omega(col, b) for b < L_nu, stored row major (b * ncols + col), and
// P(col) = Omega(col, L_nu); one thread per column, lanes over consecutive
// columns so that the U_nu loads and the Omega stores are coalesced.
template <int N, typename T>
__global__ void omega_kernel(Links<N, T> U, Geom g, ColGeom c, CField<N, T> om, CField<N, T> pol) {
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= c.ncols) return;
  const int Ln = c.Lnu;
  int x[4];
  col_coords(c, col, x);
  Mat<N, double> O = mident<N, double>();
  for (int b = 0; b < Ln; ++b) {
    om.store((long long)b * c.ncols + col, O);
    O = mul(O, to_d(U.load(site_lin(g, col_site_at(c, x, b)), c.nu)));
  }
  pol.store(col, O);
}

// U'_mu(col, row) for row < rows, over tiles of 32 consecutive columns x UP_RB
// rows: computed with lanes over columns (coalesced U and Omega reads), staged
// in shared memory and written column major (col * rows + row) with consecutive
// threads on consecutive rows.  The products run in the link precision (Omega
// itself is an FP64 product).
constexpr int UP_RB = 8;
template <int N, typename T>
__global__ void __launch_bounds__(32 * UP_RB) uprime_kernel(Links<N, T> U, Geom g, ColGeom c, CField<N, T> om,
                                                            CField<N, T> pol, CField<N, T> up) {
  __shared__ cx<T> tile[N * N][UP_RB][33];
  const long long nct = (c.ncols + 31) / 32;
  const unsigned bq = blockIdx.x / (unsigned)nct;  // the grid has fewer than 2^32 blocks
  const long long ctile = blockIdx.x - bq * (unsigned)nct;
  const int row0 = (int)bq * UP_RB;
  const int cl = threadIdx.x & 31, r = threadIdx.x >> 5;
  const long long col = ctile * 32 + cl;
  const int row = row0 + r;
  const int Ln = c.Lnu;
  if (col < c.ncols && row < c.rows) {
    const int b = row % Ln, k = row / Ln;
    int x[4];
    col_coords(c, col, x);
    const int xm = c.mu == 0 ? x[0] : c.mu == 1 ? x[1] : c.mu == 2 ? x[2] : x[3];
    const long long cp = col_shift_at(c, col, xm, 1);
    const Mat<N, T> u = U.load(site_lin(g, col_site_at(c, x, b)), c.mu);
    Mat<N, T> v = mul_nd(mul(om.load_t((long long)b * c.ncols + col), u), om.load_t((long long)b * c.ncols + cp));
    if (k > 0) {
      const Mat<N, T> P = pol.load_t(col), Pp = pol.load_t(cp);
      for (int i = 0; i < k; ++i) v = mul_nd(mul(P, v), Pp);
    }
#pragma unroll
    for (int a = 0; a < N * N; ++a) tile[a][r][cl] = v.e[a / N][a % N];
  }
  __syncthreads();
  const int cl2 = threadIdx.x / UP_RB, r2 = threadIdx.x % UP_RB;
  const long long col2 = ctile * 32 + cl2;
  const int row2 = row0 + r2;
  if (col2 < c.ncols && row2 < c.rows) {
    Mat<N, T> m;
#pragma unroll
    for (int a = 0; a < N * N; ++a) m.e[a / N][a % N] = tile[a][r2][cl2];
    up.store_t(col2 * c.rows + row2, m);
  }
}

constexpr int WL_THREADS = 128;
constexpr int WL_WARPS = WL_THREADS / 32;

// The (L, T) pair list of one launch, in the kernel parameters: entries
// off[L] .. off[L+1]-1 are the loops of spatial length L, with temporal extent
// T[k] and pair index p[k].  Up to WL_MAXP pairs and loop lengths.
struct WLTable {
  int lmax, tmax, npairs;
  int R, CW, ntile_rows;
  long long ntiles;
  short off[WL_MAXP + 2];
  short T[WL_MAXP];
  short p[WL_MAXP];
  // bit k: entries k .. k+7 have the same L and T[k+j] = T[k] + j
  uint32_t run8[WL_MAXP / 32];
};

// Sum of v[0..7] over the warp: on return lanes with (lane & 3) == 0 hold the
// total of index (lane >> 2) & 7 (a transposing butterfly: 9 shuffles, not 40).
KLFT_D double warp_transpose_sum8(double v[8], int lane) {
  const bool b16 = lane & 16, b8 = lane & 8, b4 = lane & 4;
  double w[4], x[2];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double send = b16 ? v[k] : v[k + 4];
    const double keep = b16 ? v[k + 4] : v[k];
    w[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double send = b8 ? w[k] : w[k + 2];
    const double keep = b8 ? w[k + 2] : w[k];
    x[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  const double send = b4 ? x[0] : x[1];
  double y = (b4 ? x[1] : x[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
  y += __shfl_xor_sync(0xffffffffu, y, 2);
  y += __shfl_xor_sync(0xffffffffu, y, 1);
  return y;
}

#ifndef KLFT_WL_MINB_F32
#define KLFT_WL_MINB_F32 4
#endif
template <typename T> struct WLMinBlocks { static constexpr int v = KLFT_WL_MINB_F32; };
template <> struct WLMinBlocks<double> { static constexpr int v = 2; };

// Shared tile entries are records of N*N complex numbers padded to a multiple of
// 16 bytes with an odd number of 16-byte units, so that 8 consecutive entries
// read with 16-byte loads fall in distinct bank groups (float SU(3): 80 B,
// double SU(3): 144 B).
template <int N, typename T> struct TileEnt {
  static constexpr int raw = N * N * (int)sizeof(cx<T>);
  static constexpr int r16 = (raw + 15) / 16 * 16;
  static constexpr int bytes = (r16 / 16) % 2 == 1 ? r16 : r16 + 16;
};

// Within a column's block of RT entries, even rows come first and odd rows
// after them, so that the threads of a column (which own rows 2q, 2q+1) touch
// consecutive entries: column slot of row r = (r & 1) * ((RT + 1) / 2) + (r >> 1).
KLFT_D int col_slot(int r, int half) { return (r & 1) * half + (r >> 1); }

template <int N, typename T>
KLFT_D void tile_store(unsigned char *S, int e, const Mat<N, T> &m) {
  cx<T> *q = (cx<T> *)(S + (size_t)e * TileEnt<N, T>::bytes);
#pragma unroll
  for (int k = 0; k < N * N; ++k) q[k] = m.e[k / N][k % N];
}
template <int N, typename T>
KLFT_D Mat<N, T> tile_load(const unsigned char *S, int e) {
  const cx<T> *q = (const cx<T> *)(S + (size_t)e * TileEnt<N, T>::bytes);
  Mat<N, T> m;
#pragma unroll
  for (int k = 0; k < N * N; ++k) m.e[k / N][k % N] = q[k];
  return m;
}
// Re Tr(a b^+) with b the tile entry e, in the link precision: Sum Re(a_k conj(b_k)).
template <int N, typename T>
KLFT_D T tile_trace(const Mat<N, T> &a, const unsigned char *S, int e) {
  const unsigned char *q = S + (size_t)e * TileEnt<N, T>::bytes;
  T t = T(0);
  if constexpr (sizeof(T) == 4 && (N * N) % 2 == 1) {
    // 16-byte loads of complex pairs, then the odd last one
#pragma unroll
    for (int k = 0; k + 1 < N * N; k += 2) {
      const float4 v = *(const float4 *)(q + 8 * k);
      t = fma(a.e[k / N][k % N].re, v.x, t);
      t = fma(a.e[k / N][k % N].im, v.y, t);
      t = fma(a.e[(k + 1) / N][(k + 1) % N].re, v.z, t);
      t = fma(a.e[(k + 1) / N][(k + 1) % N].im, v.w, t);
    }
    const float2 v = *(const float2 *)(q + 8 * (N * N - 1));
    t = fma(a.e[N - 1][N - 1].re, v.x, t);
    t = fma(a.e[N - 1][N - 1].im, v.y, t);
  } else {
#pragma unroll
    for (int k = 0; k < N * N; ++k) {
      const cx<T> v = ((const cx<T> *)q)[k];
      t = fma(a.e[k / N][k % N].re, v.re, t);
      t = fma(a.e[k / N][k % N].im, v.im, t);
    }
  }
  return t;
}

// Re Tr(a b^+) and Re Tr(c b^+) for one tile entry b, loaded once.
template <int N, typename T>
KLFT_D void tile_trace2(const Mat<N, T> &a, const Mat<N, T> &c, const unsigned char *S, int e, T &ta, T &tc) {
  const unsigned char *q = S + (size_t)e * TileEnt<N, T>::bytes;
  if constexpr (sizeof(T) == 4 && (N * N) % 2 == 1) {
#pragma unroll
    for (int k = 0; k + 1 < N * N; k += 2) {
      const float4 v = *(const float4 *)(q + 8 * k);
      ta = fma(a.e[k / N][k % N].re, v.x, ta);
      ta = fma(a.e[k / N][k % N].im, v.y, ta);
      ta = fma(a.e[(k + 1) / N][(k + 1) % N].re, v.z, ta);
      ta = fma(a.e[(k + 1) / N][(k + 1) % N].im, v.w, ta);
      tc = fma(c.e[k / N][k % N].re, v.x, tc);
      tc = fma(c.e[k / N][k % N].im, v.y, tc);
      tc = fma(c.e[(k + 1) / N][(k + 1) % N].re, v.z, tc);
      tc = fma(c.e[(k + 1) / N][(k + 1) % N].im, v.w, tc);
    }
    const float2 v = *(const float2 *)(q + 8 * (N * N - 1));
    ta = fma(a.e[N - 1][N - 1].re, v.x, ta);
    ta = fma(a.e[N - 1][N - 1].im, v.y, ta);
    tc = fma(c.e[N - 1][N - 1].re, v.x, tc);
    tc = fma(c.e[N - 1][N - 1].im, v.y, tc);
  } else {
#pragma unroll
    for (int k = 0; k < N * N; ++k) {
      const cx<T> v = ((const cx<T> *)q)[k];
      ta = fma(a.e[k / N][k % N].re, v.re, ta);
      ta = fma(a.e[k / N][k % N].im, v.im, ta);
      tc = fma(c.e[k / N][k % N].re, v.re, tc);
      tc = fma(c.e[k / N][k % N].im, v.im, tc);
    }
  }
}

// Persistent CTAs over tiles of CW columns x R rows; each thread owns two
// consecutive origin rows of a column.  The shared tile holds, per column, the R
// origin rows followed by T_max halo rows, so the partner of the origin at tile
// row r for extent T is entry r + T of the same column.  For a run of eight
// consecutive T the two origins share partners: 10 entry loads serve 16 traces.
template <int N, typename T>
__global__ void __launch_bounds__(WL_THREADS, WLMinBlocks<T>::v)
    wloop_kernel(CField<N, T> up, ColGeom c, const __grid_constant__ WLTable w, double *part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int RT = w.R + w.tmax;
  const int half = (RT + 1) / 2;  // entries per row parity in a column block
  const int QR = w.R / 2;          // threads per column
  double *acc = (double *)smem_raw;                                                 // [npairs][WL_WARPS]
  unsigned char *S = smem_raw + (((size_t)w.npairs * WL_WARPS * sizeof(double) + 15) & ~(size_t)15);  // entries
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int p = tid; p < w.npairs * WL_WARPS; p += WL_THREADS) acc[p] = 0.0;
  __syncthreads();
  const int Ln = c.Lnu;
  // columns never straddle a warp when QR divides 32: warp-level sync suffices
  const bool warp_local = (32 % QR) == 0;
  const bool has_origin = tid < w.CW * QR;
  const int cc = tid / QR, q = tid % QR;
  const int ebase = cc * 2 * half;
  const int eo0 = ebase + q, eo1 = ebase + half + q;  // slots of the origin rows 2q, 2q + 1
  for (long long tile = blockIdx.x; tile < w.ntiles; tile += gridDim.x) {
    const long long ctile = (long long)((unsigned)tile / (unsigned)w.ntile_rows);  // V < 2^31: 32-bit
    const int r0 = (int)(tile - ctile * w.ntile_rows) * w.R;
    const long long col = ctile * w.CW + cc;
    const bool col_ok = has_origin && col < c.ncols;
    // coordinate of the column along mu; colL = column of x + (L-1) mu, stepped per L
    const int xm = col_ok ? (int)(((unsigned)col / (unsigned)c.csmu) % (unsigned)c.Lmu) : 0;
    long long colL = col;
    int xl = xm;
    Mat<N, T> own0, own1;  // S'_L at rows r0 + 2q and r0 + 2q + 1
    for (int L = 1; L <= w.lmax; ++L) {
      if (L > 1) {
        if (++xl == c.Lmu) {
          xl = 0;
          colL -= (long long)(c.Lmu - 1) * c.csmu;
        } else {
          colL += c.csmu;
        }
      }
      if (col_ok) {
        const long long cbase = colL * c.rows + r0;
        if (r0 + 2 * q < c.rows) {
          const Mat<N, T> u = up.load_t(cbase + 2 * q);
          own0 = L == 1 ? u : mul(own0, u);
          tile_store<N, T>(S, eo0, own0);
        }
        if (r0 + 2 * q + 1 < c.rows) {
          const Mat<N, T> u = up.load_t(cbase + 2 * q + 1);
          own1 = L == 1 ? u : mul(own1, u);
          tile_store<N, T>(S, eo1, own1);
        }
        for (int j = q; j < w.tmax; j += QR) {
          if (r0 + w.R + j >= c.rows) continue;
          const int e = ebase + col_slot(w.R + j, half);
          const Mat<N, T> u = up.load_t(cbase + w.R + j);
          tile_store<N, T>(S, e, L == 1 ? u : mul(tile_load<N, T>(S, e), u));
        }
      }
      if (warp_local) __syncwarp(); else __syncthreads();
      const int k0 = w.off[L], k1 = w.off[L + 1];
      // Ln and R are even, so both origin rows are inside the axis or neither is
      const bool origin_ok = col_ok && r0 + 2 * q < Ln;
      for (int kk = k0; kk < k1; kk += 8) {
        T vt[8];
        if (kk + 8 <= k1 && ((w.run8[kk >> 5] >> (kk & 31)) & 1u)) {
          // in two halves of four extents: partner rows 2q + t0 + 4 hf + i, i = 0..4, of
          // which origin 0 takes i = 0..3 and origin 1 takes i = 1..4
#pragma unroll
          for (int hf = 0; hf < 2; ++hf) {
            const int rp = 2 * q + w.T[kk] + 4 * hf;
            T a[4], b[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) a[j] = b[j] = T(0);
            if (origin_ok) {
              a[0] = tile_trace<N, T>(own0, S, ebase + col_slot(rp, half));
#pragma unroll
              for (int i = 1; i < 4; ++i)
                tile_trace2<N, T>(own0, own1, S, ebase + col_slot(rp + i, half), a[i], b[i - 1]);
              b[3] = tile_trace<N, T>(own1, S, ebase + col_slot(rp + 4, half));
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) vt[4 * hf + j] = a[j] + b[j];
          }
        } else {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            T t = T(0);
            if (origin_ok && kk + j < k1) {
              const int rp = 2 * q + w.T[kk + j];
              t = tile_trace<N, T>(own0, S, ebase + col_slot(rp, half)) +
                  tile_trace<N, T>(own1, S, ebase + col_slot(rp + 1, half));
            }
            vt[j] = t;
          }
        }
        double v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = (double)vt[j];
        const double tot = warp_transpose_sum8(v, lane);
        const int j = (lane >> 2) & 7;
        if ((lane & 3) == 0 && kk + j < k1) acc[w.p[kk + j] * WL_WARPS + warp] += tot;
      }
      if (warp_local) __syncwarp(); else __syncthreads();
    }
  }
  __syncthreads();
  // CTA total per pair, fixed order over warps
  for (int p = tid; p < w.npairs; p += WL_THREADS) {
    double s = 0.0;
#pragma unroll
    for (int q2 = 0; q2 < WL_WARPS; ++q2) s += acc[p * WL_WARPS + q2];
    part[(long long)p * gridDim.x + blockIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
// Column-correlation form of the loop kernel (link precision FP32, every
// requested T in 1..WC_TW).  For a fixed column and loop length L,
//   sum_r W_{L,T}(col, r) = sum_r sum_k v_k(r) v_k(r + T),
// with v(r) the 2 N^2 real components of S'_L(col, r): per column it is the
// autocorrelation at lags T = 1..8 of a sequence of 2 N^2-vectors along the nu
// axis.  A CTA holds WC_CW columns x (32 origin + 8 halo) rows.  Per L each
// thread first extends the lines of two rows of its column (the running
// product S'_L = S'_{L-1} U'(x + (L-1) mu) stays in its registers) and writes
// them to shared memory component by component; after one barrier each
// "consumer" thread loads one component of a whole column (or of a chunk of
// its origin rows, for N < 3) into registers and forms all eight lags there:
// 8 x 32 FMAs per component per column from 40 shared loads, where the
// entry-per-origin form re-reads ten 3x3 entries per two origins.
constexpr int WC_TW = 8;        // lags T = 1..WC_TW
constexpr int WC_RO = 32;       // origin rows per tile
constexpr int WC_ROWS = WC_RO + WC_TW;
constexpr int WC_PT = WC_ROWS / 2;  // threads per column: two rows each
constexpr int WC_CW = 8;        // columns per CTA
constexpr int WC_THREADS = WC_PT * WC_CW;  // 160: five warps
constexpr int WC_WARPS = WC_THREADS / 32;
// Reals per component row: 44 floats (11 x 16 B) or 42 doubles (21 x 16 B),
// an odd number of 16-byte units, so that 16-byte loads of lanes a row apart
// miss each other's banks.
template <typename T> struct WCRow { static constexpr int v = 44; };
template <> struct WCRow<double> { static constexpr int v = 42; };
// CTAs per SM: the FP64 form holds twice the registers and shared memory
template <typename T> struct WCMinBlocks { static constexpr int v = 3; };
template <> struct WCMinBlocks<double> { static constexpr int v = 2; };

// Reals per column block: 2 N^2 component rows, padded (FP32) so that
// consecutive columns start 20 banks apart, and to a multiple of 16 bytes.
template <int N, typename T> struct WCCol {
  static constexpr int raw = 2 * N * N * WCRow<T>::v;
  static constexpr int v = sizeof(T) == 4 ? raw + ((20 - raw % 32 + 32) % 32) : raw + (raw & 1);
  static_assert((v * sizeof(T)) % 16 == 0, "column blocks must stay 16-byte aligned");
};
// consumer work per column: component k of origin chunk c, NCH chunks of 32 / NCH rows
template <int N> struct WCChunks { static constexpr int v = N == 3 ? 1 : N == 2 ? 2 : 8; };

// Up to WC_MAXPL planes (mu_i, nu) sharing nu in one launch: the tiles of plane
// i follow those of plane i - 1, and its U' starts pstride entries after
// plane i - 1's.
constexpr int WC_MAXPL = 3;
struct WCTable {
  int lmax, npairs, R, ntile_rows;
  long long ntiles1;  // tiles per plane
  int nplanes;
  long long pstride;
  int mu[WC_MAXPL], csmu[WC_MAXPL], Lmu[WC_MAXPL];
  short pm[WL_MAXP + 1][WC_TW];  // pair index of (L, T = j + 1), or -1
};

// Sum of v[0..7] over the warp in the lag precision: on return lanes with
// (lane & 3) == 0 hold the total of index (lane >> 2) & 7.
template <typename T> KLFT_D T warp_transpose_sum8t(T v[8], int lane) {
  const bool b16 = lane & 16, b8 = lane & 8, b4 = lane & 4;
  T w[4], x[2];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const T send = b16 ? v[k] : v[k + 4];
    const T keep = b16 ? v[k + 4] : v[k];
    w[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const T send = b8 ? w[k] : w[k + 2];
    const T keep = b8 ? w[k + 2] : w[k];
    x[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  const T send = b4 ? x[0] : x[1];
  T y = (b4 ? x[1] : x[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
  y += __shfl_xor_sync(0xffffffffu, y, 2);
  y += __shfl_xor_sync(0xffffffffu, y, 1);
  return y;
}

// a[t] += sum_{r < nv} win[r] win[r + 1 + t]; all NO origins valid when nv >= NO
template <typename T, int W, int NO>
KLFT_D void wc_lags(const T (&win)[W], T (&a)[WC_TW], int nv) {
  if (nv >= NO) {
#pragma unroll
    for (int r = 0; r < NO; ++r)
#pragma unroll
      for (int t = 0; t < WC_TW; ++t) a[t] = fma(win[r], win[r + 1 + t], a[t]);
  } else {
#pragma unroll
    for (int r = 0; r < NO; ++r) {
      const T o = r < nv ? win[r] : T(0);
#pragma unroll
      for (int t = 0; t < WC_TW; ++t) a[t] = fma(o, win[r + 1 + t], a[t]);
    }
  }
}

// W reals of a component row into registers by 16-byte loads
template <int W> KLFT_D void wc_window(const float *src, float (&win)[W]) {
#pragma unroll
  for (int i = 0; i < W / 4; ++i) {
    const float4 v = ((const float4 *)src)[i];
    win[4 * i] = v.x;
    win[4 * i + 1] = v.y;
    win[4 * i + 2] = v.z;
    win[4 * i + 3] = v.w;
  }
}
template <int W> KLFT_D void wc_window(const double *src, double (&win)[W]) {
#pragma unroll
  for (int i = 0; i < W / 2; ++i) {
    const double2 v = ((const double2 *)src)[i];
    win[2 * i] = v.x;
    win[2 * i + 1] = v.y;
  }
}

template <int N, typename T>
__global__ void __launch_bounds__(WC_THREADS, WCMinBlocks<T>::v)
    wcorr_kernel(CField<N, T> up, ColGeom c, const __grid_constant__ WCTable w, int tmax, double *part) {
  constexpr int KC = 2 * N * N;
  constexpr int NCH = WCChunks<N>::v;
  constexpr int NO = WC_RO / NCH;  // origin rows per consumer
  constexpr int W = NO + WC_TW;    // window
  constexpr int CS = WCCol<N, T>::v;
  constexpr int RS = WCRow<T>::v;
  static_assert(KC * NCH <= WC_PT, "consumer tasks must fit the threads of a column");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *buf = (T *)smem_raw;                                   // [2][WC_CW][CS]
  double *acc = (double *)(buf + 2 * WC_CW * CS);          // [nplanes * npairs][WC_WARPS]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cc = tid / WC_PT, q = tid % WC_PT;
  for (int i = tid; i < 2 * WC_CW * CS; i += WC_THREADS) buf[i] = T(0);  // rows never written stay finite
  const int nout = w.nplanes * w.npairs;
  for (int p = tid; p < nout * WC_WARPS; p += WC_THREADS) acc[p] = 0.0;
  const bool consumer = q < KC * NCH;
  const int kq = q % KC, ob = (q / KC) * NO;  // consumer's component and first origin row
  int stage = 0;
  __syncthreads();
  const long long ntiles = w.ntiles1 * w.nplanes;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // V < 2^31: tiles and columns in 32-bit arithmetic
    const int pl = (int)((unsigned)tile / (unsigned)w.ntiles1);
    const unsigned t1 = (unsigned)tile - (unsigned)pl * (unsigned)w.ntiles1;
    const long long ctile = (long long)(t1 / (unsigned)w.ntile_rows);
    const int r0 = (int)(t1 - (unsigned)ctile * (unsigned)w.ntile_rows) * w.R;
    const int reff = min(w.R, c.Lnu - r0);  // origin rows of this tile
    const int rneed = reff + tmax;           // rows read as origins or partners
    const long long col = ctile * WC_CW + cc;
    const bool col_ok = col < c.ncols;
    const int csmu = w.csmu[pl], Lmu = w.Lmu[pl];
    const int xm = col_ok ? (int)(((unsigned)col / (unsigned)csmu) % (unsigned)Lmu) : 0;
    const CField<N, T> upl{up.p + (long long)pl * w.pstride, up.n};
    double *accp = acc + (size_t)pl * w.npairs * WC_WARPS;
    long long colL = col;
    int xl = xm;
    Mat<N, T> S0, S1;  // S'_L at rows q and q + WC_PT of this column
    for (int L = 1; L <= w.lmax; ++L) {
      if (L > 1) {
        if (++xl == Lmu) {
          xl = 0;
          colL -= (long long)(Lmu - 1) * csmu;
        } else {
          colL += csmu;
        }
      }
      T *sb = buf + (stage * WC_CW + cc) * CS;
      if (col_ok && q < rneed) {
        // both rows' loads in flight before the first product
        const long long cbase = colL * c.rows + r0 + q;
        const bool two = q + WC_PT < rneed;
        const Mat<N, T> u0 = upl.load_t(cbase);
        // FP32: the second row's load too (FP64 has no registers to spare for it)
        Mat<N, T> u1;
        if constexpr (sizeof(T) == 4) u1 = two ? upl.load_t(cbase + WC_PT) : mzero<N, T>();
        S0 = L == 1 ? u0 : mul(S0, u0);
#pragma unroll
        for (int a = 0; a < N * N; ++a) {
          sb[(2 * a) * RS + q] = S0.e[a / N][a % N].re;
          sb[(2 * a + 1) * RS + q] = S0.e[a / N][a % N].im;
        }
        if (two) {
          if constexpr (sizeof(T) == 8) u1 = upl.load_t(cbase + WC_PT);
          S1 = L == 1 ? u1 : mul(S1, u1);
#pragma unroll
          for (int a = 0; a < N * N; ++a) {
            sb[(2 * a) * RS + q + WC_PT] = S1.e[a / N][a % N].re;
            sb[(2 * a + 1) * RS + q + WC_PT] = S1.e[a / N][a % N].im;
          }
        }
      }
      __syncthreads();
      T a[WC_TW];
#pragma unroll
      for (int t = 0; t < WC_TW; ++t) a[t] = T(0);
      if (consumer && col_ok) {
        if constexpr (sizeof(T) == 8 && NO % 2 == 0) {
          // FP64: the window in two halves of the origins (the overlap reloaded)
#pragma unroll 1
          for (int h = 0; h < 2; ++h) {
            T win[NO / 2 + WC_TW];
            wc_window<NO / 2 + WC_TW>(sb + kq * RS + ob + h * (NO / 2), win);
            wc_lags<T, NO / 2 + WC_TW, NO / 2>(win, a, reff - ob - h * (NO / 2));
          }
        } else {
          T win[W];
          wc_window<W>(sb + kq * RS + ob, win);
          wc_lags<T, W, NO>(win, a, reff - ob);
        }
      }
      const T tot = warp_transpose_sum8t<T>(a, lane);
      const int j = (lane >> 2) & 7;
      if ((lane & 3) == 0) {
        const int p = w.pm[L][j];
        if (p >= 0) accp[p * WC_WARPS + warp] += (double)tot;
      }
      stage ^= 1;
    }
  }
  __syncthreads();
  for (int p = tid; p < nout; p += WC_THREADS) {
    double s = 0.0;
#pragma unroll
    for (int q2 = 0; q2 < WC_WARPS; ++q2) s += acc[p * WC_WARPS + q2];
    part[(long long)p * gridDim.x + blockIdx.x] = s;
  }
}

template <int N, typename T> static size_t wcorr_smem(int npairs) {
  return (size_t)2 * WC_CW * WCCol<N, T>::v * sizeof(T) + (size_t)npairs * WC_WARPS * sizeof(double);
}

// Whether the column-correlation kernel serves this table: every T in 1..WC_TW.
static bool wcorr_eligible(int tmax, const int *T, int nent) {
  if (tmax > WC_TW) return false;
  for (int k = 0; k < nent; ++k)
    if (T[k] < 1 || T[k] > WC_TW) return false;
  return true;
}

// Scratch needed by launch_wilson_gf (bytes).
size_t wilson_gf_scratch(int nc, int dtype, const Geom &g, int nu, int tmax, int nplanes) {
  // bytes per site of a scratch field (CField: FP32 entries in 16-byte pairs)
  const size_t es = dtype == 0 ? 16 * (size_t)nc * nc : 16 * (size_t)((nc * nc + 1) / 2);
  const size_t rows = (size_t)g.L[nu] + (size_t)tmax;
  const size_t ncols = (size_t)(g.V / g.L[nu]);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  // Omega, P, and one U' per plane
  return al(es * g.V) + al(es * ncols) + (size_t)nplanes * al(es * ncols * rows);
}

// R origin rows per column tile (even: each thread owns two), CW columns per CTA.
static void tile_shape(const Geom &g, int nu, int &R, int &CW) {
  const int Ln = g.L[nu];
  R = Ln < 32 ? Ln : 32;
  CW = WL_THREADS / (R / 2);
}

static size_t tile_entry_bytes(int nc, int dtype) {
  if (dtype == 0) return nc == 1 ? TileEnt<1, double>::bytes : nc == 2 ? TileEnt<2, double>::bytes : TileEnt<3, double>::bytes;
  return nc == 1 ? TileEnt<1, float>::bytes : nc == 2 ? TileEnt<2, float>::bytes : TileEnt<3, float>::bytes;
}

size_t wilson_gf_smem(int nc, int dtype, const Geom &g, int nu, int tmax, int npairs) {
  int R, CW;
  tile_shape(g, nu, R, CW);
  return (((size_t)npairs * WL_WARPS * sizeof(double) + 15) & ~(size_t)15) +
         tile_entry_bytes(nc, dtype) * (size_t)CW * (2 * ((R + tmax + 1) / 2));
}

int wilson_gf_blocks(const Geom &g) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  (void)g;
  return sms * 4;
}

// The loops of nplanes planes (mus[i], nu) that share nu: one Omega, one U' per
// plane, then the loop kernel; plane i's partial sums at d_part[(i * npairs + k) * grid + b].
template <int N, typename T>
static cudaError_t wilson_gf_t(const void *links, const Geom &g, const int *const *h_tab, int lmax, int tmax,
                               int npairs, const int *mus, int nplanes, int nu, bool omega_ready, void *scratch,
                               double *d_part, int nblk, int *grid_used, cudaStream_t st, cudaStream_t stl,
                               cudaEvent_t ev) {
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  if (nplanes < 1 || nplanes > WC_MAXPL) return cudaErrorInvalidValue;
  if (npairs > WL_MAXP || lmax > WL_MAXP || tmax > 32767) return cudaErrorInvalidValue;
  const size_t es = CField<N, T>::bytes(1);
  ColGeom c[WC_MAXPL];
  for (int i = 0; i < nplanes; ++i) c[i] = make_colgeom(g, mus[i], nu, g.L[nu] + tmax);
  const long long Vc = c[0].ncols * g.L[nu];
  const size_t up_bytes = al(es * c[0].ncols * c[0].rows);
  char *base = (char *)scratch;
  CField<N, T> om{(cx<T> *)base, Vc};
  CField<N, T> pol{(cx<T> *)(base + al(es * Vc)), c[0].ncols};
  char *up0 = base + al(es * Vc) + al(es * c[0].ncols);
  Links<N, T> U{(cx<T> *)links, g.V};
  if (!omega_ready) omega_kernel<N, T><<<(unsigned)((c[0].ncols + 127) / 128), 128, 0, st>>>(U, g, c[0], om, pol);
  const long long nct = (c[0].ncols + 31) / 32;
  for (int i = 0; i < nplanes; ++i) {
    const CField<N, T> up{(cx<T> *)(up0 + i * up_bytes), c[i].ncols * c[i].rows};
    uprime_kernel<N, T><<<(unsigned)(nct * ((c[i].rows + UP_RB - 1) / UP_RB)), 32 * UP_RB, 0, st>>>(U, g, c[i], om,
                                                                                                 pol, up);
  }
  // the loop kernels read U' only: on stl (if given) after U' is complete
  if (stl) {
    cudaError_t e = cudaEventRecord(ev, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stl, ev, 0);
    if (e != cudaSuccess) return e;
    st = stl;
  }
  const CField<N, T> up{(cx<T> *)up0, c[0].ncols * c[0].rows};
  if (wcorr_eligible(tmax, h_tab[1], h_tab[0][lmax + 1])) {
    WCTable w;
    std::memset(&w, 0, sizeof w);
    w.lmax = lmax;
    w.npairs = npairs;
    for (int L = 0; L <= WL_MAXP; ++L)
      for (int j = 0; j < WC_TW; ++j) w.pm[L][j] = -1;
    bool dup = false;
    for (int L = 1; L <= lmax; ++L)
      for (int k = h_tab[0][L]; k < h_tab[0][L + 1]; ++k) {
        short &m = w.pm[L][h_tab[1][k] - 1];
        dup = dup || m >= 0;
        m = (short)h_tab[2][k];
      }
    if (!dup) {
      w.R = g.L[nu] < WC_RO ? g.L[nu] : WC_RO;
      w.ntile_rows = (g.L[nu] + w.R - 1) / w.R;
      w.ntiles1 = ((c[0].ncols + WC_CW - 1) / WC_CW) * w.ntile_rows;
      w.nplanes = nplanes;
      w.pstride = (long long)(up_bytes / sizeof(cx<T>));
      for (int i = 0; i < nplanes; ++i) {
        w.mu[i] = mus[i];
        w.csmu[i] = c[i].csmu;
        w.Lmu[i] = c[i].Lmu;
      }
      const size_t smem = wcorr_smem<N, T>(npairs * nplanes);
      // the attribute is per device: set it on every launch
      cudaFuncSetAttribute(wcorr_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 120 * 1024);
      // resident CTAs on the device, queried once per (N, T) (thread-safe static initialisation)
      static const long long want = [] {
        int dev = 0, sms = 0, nb = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, wcorr_kernel<N, T>, WC_THREADS,
                                                      wcorr_smem<N, T>(WL_MAXP * WC_MAXPL));
        return (long long)(sms > 0 ? sms : 148) * (nb > 0 ? nb : 1);
      }();
      const long long ntiles = w.ntiles1 * nplanes;
      const int grid = (int)std::min<long long>(std::min<long long>(want, nblk), ntiles > 0 ? ntiles : 1);
      wcorr_kernel<N, T><<<grid, WC_THREADS, smem, st>>>(up, c[0], w, tmax, d_part);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      *grid_used = grid;
      return cudaSuccess;
    }
  }
  // entry-per-origin kernel: one launch per plane
  WLTable w;
  std::memset(&w, 0, sizeof w);
  w.lmax = lmax;
  w.tmax = tmax;
  w.npairs = npairs;
  for (int L = 0; L <= lmax + 1; ++L) w.off[L] = (short)h_tab[0][L];
  for (int k = 0; k < npairs; ++k) {
    w.T[k] = (short)h_tab[1][k];
    w.p[k] = (short)h_tab[2][k];
  }
  for (int L = 1; L <= lmax; ++L)
    for (int k = h_tab[0][L]; k + 8 <= h_tab[0][L + 1]; ++k) {
      bool run = true;
      for (int j = 1; j < 8; ++j) run = run && h_tab[1][k + j] == h_tab[1][k] + j;
      if (run) w.run8[k >> 5] |= 1u << (k & 31);
    }
  tile_shape(g, nu, w.R, w.CW);
  w.ntile_rows = (g.L[nu] + w.R - 1) / w.R;
  w.ntiles = ((c[0].ncols + w.CW - 1) / w.CW) * w.ntile_rows;
  const size_t smem = (((size_t)npairs * WL_WARPS * sizeof(double) + 15) & ~(size_t)15) +
                      (size_t)TileEnt<N, T>::bytes * w.CW * (2 * ((w.R + tmax + 1) / 2));
  cudaFuncSetAttribute(wloop_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  for (int i = 0; i < nplanes; ++i) {
    const CField<N, T> upi{(cx<T> *)(up0 + i * up_bytes), c[i].ncols * c[i].rows};
    wloop_kernel<N, T><<<nblk, WL_THREADS, smem, st>>>(upi, c[i], w, d_part + (size_t)i * npairs * nblk);
  }
  *grid_used = nblk;
  return cudaGetLastError();
}

cudaError_t launch_wilson_gf(int nc, int dtype, const void *links, const Geom &g, const int *mus, int nplanes,
                             int nu, const int *const *h_tab, int lmax, int tmax, int npairs, bool omega_ready,
                             void *scratch, double *d_part, int nblk, double *d_out, int out_stride,
                             cudaStream_t st, cudaStream_t st_loops, cudaEvent_t ev) {
  cudaError_t e = cudaErrorInvalidValue;
  if (st_loops && !ev) return e;
  int grid = nblk;  // CTAs that wrote partial sums
#define KLFT_WGF(NV, TV)                                                                                        \
  e = wilson_gf_t<NV, TV>(links, g, h_tab, lmax, tmax, npairs, mus, nplanes, nu, omega_ready, scratch, d_part, \
                          nblk, &grid, st, st_loops, ev)
  if (dtype == 0) {
    if (nc == 1) KLFT_WGF(1, double);
    else if (nc == 2) KLFT_WGF(2, double);
    else if (nc == 3) KLFT_WGF(3, double);
  } else {
    if (nc == 1) KLFT_WGF(1, float);
    else if (nc == 2) KLFT_WGF(2, float);
    else if (nc == 3) KLFT_WGF(3, float);
  }
#undef KLFT_WGF
  if (e != cudaSuccess) return e;
  if (st_loops) st = st_loops;
  // plane i's sums at d_out + i * out_stride: one reduction launch when they are contiguous
  if (out_stride == npairs) return launch_reduce_partials(d_part, grid, nplanes * npairs, d_out, st);
  for (int i = 0; i < nplanes && e == cudaSuccess; ++i)
    e = launch_reduce_partials(d_part + (size_t)i * npairs * grid, grid, npairs, d_out + (size_t)i * out_stride, st);
  return e;
}

}  // namespace klft
