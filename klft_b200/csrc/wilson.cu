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
// Kernels: omega_kernel (per nu: the axial-gauge transformation, FP64),
// uprime_kernel (per plane: U'_mu on L_nu + T_max rows, computed in FP64 and
// stored in the link precision), wloop_kernel (per plane: persistent CTAs over
// tiles of CW columns x R rows; S'_L is built incrementally over L in shared
// memory together with a halo of T_max rows of the same column; per-site traces
// in the link precision, lattice sums in FP64).
//
// Omega and U' are stored "column major": entry (column c, row b) at c*rows + b,
// one plane per complex colour entry, so a warp covering consecutive rows of
// one column reads contiguous memory.
#include "common.cuh"
#include "kernels.cuh"

namespace klft {

struct ColGeom {
  int nd, mu, nu;
  int L[4];
  int cs[4];      // column stride of each dimension (0 for nu)
  long long ncols;
  int rows;       // stored rows of U' (L_nu + extension)
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
  return c;
}

// site of (column, row) with row < L_nu
KLFT_D Site col_site(const ColGeom &c, long long col, int row) {
  Site s;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    int x;
    if (d == c.nu) {
      x = row;
    } else if (d < c.nd) {
      x = (int)(col % c.L[d]);
      col /= c.L[d];
    } else {
      x = 0;
    }
    s.b[d] = x & 1;
    s.h[d] = x >> 1;
  }
  return s;
}

// column index of xbar + k mu
KLFT_D long long col_shift(const ColGeom &c, long long col, int k) {
  const int Lm = c.L[c.mu];
  const int xm = (int)((col / c.cs[c.mu]) % Lm);
  const int xn = (xm + k) % Lm;
  return col + (long long)(xn - xm) * c.cs[c.mu];
}

template <int N, typename T> struct CField {
  cx<T> *p;
  long long n;  // entries per colour plane
  KLFT_D Mat<N, double> load(long long i) const {
    Mat<N, double> m;
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int b = 0; b < N; ++b) {
        const cx<T> v = p[(a * N + b) * n + i];
        m.e[a][b] = mk<double>((double)v.re, (double)v.im);
      }
    return m;
  }
  KLFT_D Mat<N, T> load_t(long long i) const {
    Mat<N, T> m;
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int b = 0; b < N; ++b) m.e[a][b] = p[(a * N + b) * n + i];
    return m;
  }
  KLFT_D void store(long long i, const Mat<N, double> &m) const {
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int b = 0; b < N; ++b) p[(a * N + b) * n + i] = mk<T>((T)m.e[a][b].re, (T)m.e[a][b].im);
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

// Omega(col, b) for b < L_nu, and P(col) = Omega(col, L_nu); one thread per column.
template <int N, typename T>
__global__ void omega_kernel(Links<N, T> U, Geom g, ColGeom c, CField<N, T> om, CField<N, T> pol) {
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= c.ncols) return;
  const int Ln = c.L[c.nu];
  Mat<N, double> O = mident<N, double>();
  for (int b = 0; b < Ln; ++b) {
    om.store(col * Ln + b, O);
    O = mul(O, to_d(U.load(site_lin(g, col_site(c, col, b)), c.nu)));
  }
  pol.store(col, O);
}

// U'_mu(col, row) for row < rows; one thread per entry, rows fastest.  The
// products run in the link precision (Omega itself is an FP64 product).
template <int N, typename T>
__global__ void __launch_bounds__(128) uprime_kernel(Links<N, T> U, Geom g, ColGeom c, CField<N, T> om,
                                                     CField<N, T> pol, CField<N, T> up) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= c.ncols * c.rows) return;
  const long long col = t / c.rows;
  const int row = (int)(t - col * c.rows);
  const int Ln = c.L[c.nu];
  const int b = row % Ln, k = row / Ln;
  const long long cp = col_shift(c, col, 1);
  const Mat<N, T> u = U.load(site_lin(g, col_site(c, col, b)), c.mu);
  Mat<N, T> v = mul_nd(mul(om.load_t(col * Ln + b), u), om.load_t(cp * Ln + b));
  if (k > 0) {
    const Mat<N, T> P = pol.load_t(col), Pp = pol.load_t(cp);
    for (int i = 0; i < k; ++i) v = mul_nd(mul(P, v), Pp);
  }
#pragma unroll
  for (int a = 0; a < N; ++a)
#pragma unroll
    for (int bb = 0; bb < N; ++bb) up.p[(a * N + bb) * up.n + t] = v.e[a][bb];
}

constexpr int WL_THREADS = 128;
constexpr int WL_WARPS = WL_THREADS / 32;

struct WLTable {
  int lmax, tmax, npairs;
  int R, CW, ntile_rows;
  long long ntiles;
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

// Loops for all requested (L, T): tab_off[L]..tab_off[L+1] index tab_T / tab_p.
template <typename T> struct WLMinBlocks { static constexpr int v = 4; };
template <> struct WLMinBlocks<double> { static constexpr int v = 2; };

template <int N, typename T>
__global__ void __launch_bounds__(WL_THREADS, WLMinBlocks<T>::v) wloop_kernel(CField<N, T> up, ColGeom c, WLTable w,
                                                           const int *__restrict__ tab_off,
                                                           const int *__restrict__ tab_T,
                                                           const int *__restrict__ tab_p, double *part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int E = w.CW * (w.R + w.tmax);  // entries: origins first, then halo rows
  double *acc = (double *)smem_raw;                          // [npairs][WL_WARPS]
  cx<T> *S = (cx<T> *)(acc + (size_t)w.npairs * WL_WARPS);  // [N*N][E]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int p = tid; p < w.npairs * WL_WARPS; p += WL_THREADS) acc[p] = 0.0;
  __syncthreads();
  const int Ln = c.L[c.nu];
  const int norig = w.CW * w.R;
  // columns never straddle a warp when R divides 32: warp-level sync suffices
  const bool warp_local = (32 % w.R) == 0;
  const bool has_origin = tid < norig;
  const int cc = tid / w.R, rr = tid % w.R;
  for (long long tile = blockIdx.x; tile < w.ntiles; tile += gridDim.x) {
    const long long ctile = tile / w.ntile_rows;
    const int r0 = (int)(tile - ctile * w.ntile_rows) * w.R;
    const long long col = ctile * w.CW + cc;
    const bool col_ok = has_origin && col < c.ncols;
    Mat<N, T> own;  // S'_L at (col, r0 + rr)
    for (int L = 1; L <= w.lmax; ++L) {
      if (col_ok) {
        const long long colL = col_shift(c, col, L - 1);
        // own origin entry
        {
          const int row = r0 + rr;
          if (row < c.rows) {
            const Mat<N, T> u = up.load_t(colL * c.rows + row);
            own = L == 1 ? u : mul(own, u);
#pragma unroll
            for (int a = 0; a < N * N; ++a) S[a * E + tid] = own.e[a / N][a % N];
          }
        }
        // halo entries j = rr, rr + R, ... of this column
        for (int j = rr; j < w.tmax; j += w.R) {
          const int row = r0 + w.R + j;
          const int e = norig + cc * w.tmax + j;
          if (row >= c.rows) continue;
          const Mat<N, T> u = up.load_t(colL * c.rows + row);
          Mat<N, T> s;
          if (L == 1) {
            s = u;
          } else {
            Mat<N, T> prev;
#pragma unroll
            for (int a = 0; a < N * N; ++a) prev.e[a / N][a % N] = S[a * E + e];
            s = mul(prev, u);
          }
#pragma unroll
          for (int a = 0; a < N * N; ++a) S[a * E + e] = s.e[a / N][a % N];
        }
      }
      if (warp_local) __syncwarp(); else __syncthreads();
      const int k0 = tab_off[L], k1 = tab_off[L + 1];
      const bool origin_ok = col_ok && r0 + rr < Ln;
      for (int kk = k0; kk < k1; kk += 8) {
        const int cnt = k1 - kk < 8 ? k1 - kk : 8;
        double v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          v[j] = 0.0;
          if (origin_ok && j < cnt) {
            const int rr2 = rr + tab_T[kk + j];
            const int e2 = rr2 < w.R ? cc * w.R + rr2 : norig + cc * w.tmax + (rr2 - w.R);
            // the trace of one loop in the link precision
            T t = T(0);
#pragma unroll
            for (int a = 0; a < N * N; ++a) {
              const cx<T> o = own.e[a / N][a % N], q = S[a * E + e2];
              t += o.re * q.re + o.im * q.im;
            }
            v[j] = (double)t;
          }
        }
        const double tot = warp_transpose_sum8(v, lane);
        const int j = (lane >> 2) & 7;
        if ((lane & 3) == 0 && j < cnt) acc[tab_p[kk + j] * WL_WARPS + warp] += tot;
      }
      if (warp_local) __syncwarp(); else __syncthreads();
    }
  }
  __syncthreads();
  // CTA total per pair, fixed order over warps
  for (int p = tid; p < w.npairs; p += WL_THREADS) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < WL_WARPS; ++q) s += acc[p * WL_WARPS + q];
    part[(long long)p * gridDim.x + blockIdx.x] = s;
  }
}

// Scratch needed by launch_wilson_gf (bytes).
size_t wilson_gf_scratch(int nc, int dtype, const Geom &g, int nu, int tmax) {
  const size_t es = (dtype == 0 ? 16 : 8) * (size_t)nc * nc;
  const size_t rows = (size_t)g.L[nu] + (size_t)tmax;
  const size_t ncols = (size_t)(g.V / g.L[nu]);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  return al(es * g.V) + al(es * ncols) + al(es * ncols * rows);
}

static void tile_shape(const Geom &g, int nu, int &R, int &CW) {
  const int Ln = g.L[nu];
  R = Ln < 32 ? Ln : 32;
  CW = WL_THREADS / R;
}

size_t wilson_gf_smem(int nc, int dtype, const Geom &g, int nu, int tmax, int npairs) {
  const size_t es = (dtype == 0 ? 16 : 8) * (size_t)nc * nc;
  int R, CW;
  tile_shape(g, nu, R, CW);
  return (size_t)npairs * WL_WARPS * sizeof(double) + es * (size_t)CW * (R + tmax);
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

template <int N, typename T>
static cudaError_t wilson_gf_t(const void *links, const Geom &g, const int *const *d_tab, int lmax, int tmax,
                               int npairs, int mu, int nu, bool omega_ready, void *scratch, double *d_part, int nblk,
                               cudaStream_t st) {
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t es = sizeof(cx<T>) * N * N;
  const ColGeom c = make_colgeom(g, mu, nu, g.L[nu] + tmax);
  const long long Vc = c.ncols * g.L[nu];
  char *base = (char *)scratch;
  CField<N, T> om{(cx<T> *)base, Vc};
  CField<N, T> pol{(cx<T> *)(base + al(es * Vc)), c.ncols};
  CField<N, T> up{(cx<T> *)(base + al(es * Vc) + al(es * c.ncols)), c.ncols * c.rows};
  Links<N, T> U{(cx<T> *)links, g.V};
  if (!omega_ready) omega_kernel<N, T><<<(unsigned)((c.ncols + 127) / 128), 128, 0, st>>>(U, g, c, om, pol);
  uprime_kernel<N, T><<<(unsigned)((c.ncols * c.rows + 127) / 128), 128, 0, st>>>(U, g, c, om, pol, up);
  WLTable w;
  w.lmax = lmax;
  w.tmax = tmax;
  w.npairs = npairs;
  tile_shape(g, nu, w.R, w.CW);
  w.ntile_rows = (g.L[nu] + w.R - 1) / w.R;
  w.ntiles = ((c.ncols + w.CW - 1) / w.CW) * w.ntile_rows;
  const size_t smem = (size_t)npairs * WL_WARPS * sizeof(double) + es * (size_t)w.CW * (w.R + tmax);
  cudaFuncSetAttribute(wloop_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  wloop_kernel<N, T><<<nblk, WL_THREADS, smem, st>>>(up, c, w, d_tab[0], d_tab[1], d_tab[2], d_part);
  return cudaGetLastError();
}

cudaError_t launch_wilson_gf(int nc, int dtype, const void *links, const Geom &g, int mu, int nu,
                             const int *const *d_tab, const int *h_off, int lmax, int tmax, int npairs,
                             bool omega_ready, void *scratch, double *d_part, int nblk, double *d_out,
                             cudaStream_t st) {
  (void)h_off;
  cudaError_t e = cudaErrorInvalidValue;
#define KLFT_WGF(NV, TV) \
  e = wilson_gf_t<NV, TV>(links, g, d_tab, lmax, tmax, npairs, mu, nu, omega_ready, scratch, d_part, nblk, st)
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
  return launch_reduce_partials(d_part, nblk, npairs, d_out, st);
}

}  // namespace klft
