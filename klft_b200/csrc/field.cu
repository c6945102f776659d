// field.cu -- link-field utility kernels: cold/hot start, conversion between the
// host interchange layout (AoS FP64, x0 fastest) and the device layout,
// reunitarisation, the unitarity monitor and the all-links staple field.
#include "group.cuh"
#include "kernels.cuh"
#include "staple.cuh"

namespace klft {

// deviceGaugeField init ctors (GaugeField.hpp:65-141): cold = identity
// (lib/Metropolis.cpp:79-81); hot = Haar-random link from the (site, mu) stream.
template <int NC, typename T>
__global__ void init_kernel(Links<NC, T> U, Geom g, int hot, uint64_t seed, uint64_t chain) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const long long lex = t / g.nd;
  const int mu = (int)(t - lex * g.nd);
  const Site s = site_from_lex(g, lex);
  Mat<NC, T> m = mident<NC, T>();
  if (hot) {
    Stream st(seed, chain, (uint32_t)lex, 0u, KIND_INIT, (uint32_t)mu);
    m = haar<T>(st, (const Mat<NC, T> *)nullptr);
  }
  U.store(site_lin(g, s), mu, m);
}

template <int NC, typename T>
__global__ void import_kernel(Links<NC, T> U, Geom g, const double *__restrict__ aos) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const long long lex = t / g.nd;
  const int mu = (int)(t - lex * g.nd);
  const double *p = aos + t * (2 * NC * NC);
  Mat<NC, T> m;
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) m.e[i][j] = mk<T>((T)p[2 * (i * NC + j)], (T)p[2 * (i * NC + j) + 1]);
  U.store(site_lin(g, site_from_lex(g, lex)), mu, m);
}

template <int NC, typename T>
__global__ void export_kernel(Links<NC, T> U, Geom g, double *__restrict__ aos) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const long long lex = t / g.nd;
  const int mu = (int)(t - lex * g.nd);
  const Mat<NC, T> m = U.load(site_lin(g, site_from_lex(g, lex)), mu);
  double *p = aos + t * (2 * NC * NC);
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) {
      p[2 * (i * NC + j)] = (double)m.e[i][j].re;
      p[2 * (i * NC + j) + 1] = (double)m.e[i][j].im;
    }
}

// Mixed form: the stored FP32 reals of each link in the interchange order
// (link t = lex * Nd + mu holds F = 2 LinkPlanes reals at t * F), the first F
// of its 2 N^2 interchange values.
template <int NC>
__global__ void import_f32_kernel(Links<NC, float> U, Geom g, const float *__restrict__ aos) {
  constexpr int P = Links<NC, float>::P;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const long long lex = t / g.nd;
  const int mu = (int)(t - lex * g.nd);
  const float *p = aos + t * (2 * P);
  cx<float> *q = U.p + (long long)mu * P * U.V + site_lin(g, site_from_lex(g, lex));
#pragma unroll
  for (int k = 0; k < P; ++k) q[k * U.V] = mk<float>(p[2 * k], p[2 * k + 1]);
}

template <int NC>
__global__ void export_f32_kernel(Links<NC, float> U, Geom g, float *__restrict__ aos) {
  constexpr int P = Links<NC, float>::P;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const long long lex = t / g.nd;
  const int mu = (int)(t - lex * g.nd);
  float *p = aos + t * (2 * P);
  const cx<float> *q = U.p + (long long)mu * P * U.V + site_lin(g, site_from_lex(g, lex));
#pragma unroll
  for (int k = 0; k < P; ++k) {
    const cx<float> v = q[k * U.V];
    p[2 * k] = v.re;
    p[2 * k + 1] = v.im;
  }
}

// restoreSUN on every link; the mixed form reunitarises in FP64
template <int NC, typename T>
__global__ void reunitarize_kernel(Links<NC, T> U, Geom g) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * g.nd) return;
  const int mu = (int)(t / g.V);
  const long long lin = t - (long long)mu * g.V;
  if (g.open_mu == mu && open_link(g, site_from_lin(g, lin), mu)) return;
  const Mat<NC, T> m = U.load(lin, mu);
  Mat<NC, double> d;
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) d.e[i][j] = mk<double>((double)m.e[i][j].re, (double)m.e[i][j].im);
  d = restore(d);
  Mat<NC, T> o;
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) o.e[i][j] = mk<T>((T)d.e[i][j].re, (T)d.e[i][j].im);
  U.store(lin, mu, o);
}

// open boundary in direction g.open_mu: zero the links on the last slice
template <int NC, typename T>
__global__ void open_boundary_kernel(Links<NC, T> U, Geom g) {
  const long long lin = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (lin >= g.V) return;
  if (!open_link(g, site_from_lin(g, lin), g.open_mu)) return;
  U.store(lin, g.open_mu, mzero<NC, T>());
}

template <int NC, typename T>
__global__ void unitarity_kernel(Links<NC, T> U, Geom g, double *part) {
  double worst = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < g.V * g.nd;
       t += (long long)gridDim.x * blockDim.x) {
    const int mu = (int)(t / g.V);
    const long long lin = t - (long long)mu * g.V;
    if (g.open_mu == mu && open_link(g, site_from_lin(g, lin), mu)) continue;
    const Mat<NC, T> m = U.load(lin, mu);
    Mat<NC, double> d;
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) d.e[i][j] = mk<double>((double)m.e[i][j].re, (double)m.e[i][j].im);
    const Mat<NC, double> p = mul_dn(d, d);
    double e = 0.0;
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
      for (int j = 0; j < NC; ++j) {
        const double re = p.e[i][j].re - (i == j ? 1.0 : 0.0), im = p.e[i][j].im;
        e += re * re + im * im;
      }
    worst = fmax(worst, sqrt(e));
  }
  __shared__ double red[256];
  red[threadIdx.x] = worst;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void max_partials_kernel(const double *part, int n, double *out) {
  __shared__ double red[256];
  double w = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) w = fmax(w, part[i]);
  red[threadIdx.x] = w;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// Gauge_Util.hpp:27-97 stapleField: the staple of every (x, mu), in host layout
template <int NC, int ND, typename T>
__global__ void staple_field_kernel(Links<NC, T> U, Geom g, double *__restrict__ aos) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.V * ND) return;
  const long long lex = t / ND;
  const int mu = (int)(t - lex * ND);
  const Site x = site_from_lex(g, lex);
  Defect none{0, 1, {0, 0, 0}, 1.0, nullptr};
  const Mat<NC, T> S = staple<NC, ND, T>(U, g, x, mu, none);
  double *p = aos + t * (2 * NC * NC);
#pragma unroll
  for (int i = 0; i < NC; ++i)
#pragma unroll
    for (int j = 0; j < NC; ++j) {
      p[2 * (i * NC + j)] = (double)S.e[i][j].re;
      p[2 * (i * NC + j) + 1] = (double)S.e[i][j].im;
    }
}

#define KLFT_DISPATCH_NC_T(nc, dtype, CALL)                        \
  do {                                                            \
    if (dtype == 0) {                                             \
      if (nc == 1) { using T = double; constexpr int NC = 1; CALL; } \
      else if (nc == 2) { using T = double; constexpr int NC = 2; CALL; } \
      else if (nc == 3) { using T = double; constexpr int NC = 3; CALL; } \
      else return cudaErrorInvalidValue;                          \
    } else {                                                      \
      if (nc == 1) { using T = float; constexpr int NC = 1; CALL; } \
      else if (nc == 2) { using T = float; constexpr int NC = 2; CALL; } \
      else if (nc == 3) { using T = float; constexpr int NC = 3; CALL; } \
      else return cudaErrorInvalidValue;                          \
    }                                                             \
  } while (0)

static inline unsigned nblocks(long long n, int b) { return (unsigned)((n + b - 1) / b); }

cudaError_t launch_init(int nc, int dtype, void *links, const Geom &g, int hot, uint64_t seed, uint64_t chain,
                        cudaStream_t st) {
  KLFT_DISPATCH_NC_T(nc, dtype, (init_kernel<NC, T><<<nblocks(g.V * g.nd, 256), 256, 0, st>>>(
                                    Links<NC, T>{(cx<T> *)links, g.V}, g, hot, seed, chain)));
  return cudaGetLastError();
}

cudaError_t launch_import(int nc, int dtype, void *links, const Geom &g, const double *aos, cudaStream_t st) {
  KLFT_DISPATCH_NC_T(nc, dtype, (import_kernel<NC, T><<<nblocks(g.V * g.nd, 256), 256, 0, st>>>(
                                    Links<NC, T>{(cx<T> *)links, g.V}, g, aos)));
  return cudaGetLastError();
}

cudaError_t launch_import_f32(int nc, void *links, const Geom &g, const float *aos, cudaStream_t st) {
  const unsigned nb = nblocks(g.V * g.nd, 256);
  if (nc == 1) import_f32_kernel<1><<<nb, 256, 0, st>>>(Links<1, float>{(cx<float> *)links, g.V}, g, aos);
  else if (nc == 2) import_f32_kernel<2><<<nb, 256, 0, st>>>(Links<2, float>{(cx<float> *)links, g.V}, g, aos);
  else if (nc == 3) import_f32_kernel<3><<<nb, 256, 0, st>>>(Links<3, float>{(cx<float> *)links, g.V}, g, aos);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_export_f32(int nc, const void *links, const Geom &g, float *aos, cudaStream_t st) {
  const unsigned nb = nblocks(g.V * g.nd, 256);
  if (nc == 1) export_f32_kernel<1><<<nb, 256, 0, st>>>(Links<1, float>{(cx<float> *)links, g.V}, g, aos);
  else if (nc == 2) export_f32_kernel<2><<<nb, 256, 0, st>>>(Links<2, float>{(cx<float> *)links, g.V}, g, aos);
  else if (nc == 3) export_f32_kernel<3><<<nb, 256, 0, st>>>(Links<3, float>{(cx<float> *)links, g.V}, g, aos);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_export(int nc, int dtype, const void *links, const Geom &g, double *aos, cudaStream_t st) {
  KLFT_DISPATCH_NC_T(nc, dtype, (export_kernel<NC, T><<<nblocks(g.V * g.nd, 256), 256, 0, st>>>(
                                    Links<NC, T>{(cx<T> *)links, g.V}, g, aos)));
  return cudaGetLastError();
}

cudaError_t launch_reunitarize(int nc, int dtype, void *links, const Geom &g, cudaStream_t st) {
  KLFT_DISPATCH_NC_T(nc, dtype, (reunitarize_kernel<NC, T><<<nblocks(g.V * g.nd, 256), 256, 0, st>>>(
                                    Links<NC, T>{(cx<T> *)links, g.V}, g)));
  return cudaGetLastError();
}

cudaError_t launch_open_boundary(int nc, int dtype, void *links, const Geom &g, cudaStream_t st) {
  if (g.open_mu < 0) return cudaSuccess;
  KLFT_DISPATCH_NC_T(nc, dtype, (open_boundary_kernel<NC, T><<<nblocks(g.V, 256), 256, 0, st>>>(
                                    Links<NC, T>{(cx<T> *)links, g.V}, g)));
  return cudaGetLastError();
}

cudaError_t launch_unitarity(int nc, int dtype, const void *links, const Geom &g, double *d_part, double *d_out,
                             cudaStream_t st) {
  const int nb = 296;
  KLFT_DISPATCH_NC_T(nc, dtype, (unitarity_kernel<NC, T><<<nb, 256, 0, st>>>(
                                    Links<NC, T>{(cx<T> *)links, g.V}, g, d_part)));
  max_partials_kernel<<<1, 256, 0, st>>>(d_part, nb, d_out);
  return cudaGetLastError();
}

cudaError_t launch_staple_field(int nc, int dtype, const void *links, const Geom &g, double *aos, cudaStream_t st) {
  const unsigned nb = nblocks(g.V * g.nd, 128);
#define KLFT_SF(NDV) staple_field_kernel<NC, NDV, T><<<nb, 128, 0, st>>>(Links<NC, T>{(cx<T> *)links, g.V}, g, aos)
  KLFT_DISPATCH_NC_T(nc, dtype, ({
    if (g.nd == 2) KLFT_SF(2);
    else if (g.nd == 3) KLFT_SF(3);
    else KLFT_SF(4);
  }));
#undef KLFT_SF
  return cudaGetLastError();
}

}  // namespace klft
