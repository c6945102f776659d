// hostio.cu -- host <-> device copies of whole lattices (klft_lattice_upload /
// klft_lattice_download; GaugeField.hpp:30-141 keeps its fields in host-visible
// Kokkos views, so callers of the reference hand configurations around as host
// arrays).
//
// A host buffer that is page-locked (cudaHostAlloc / cudaHostRegister) is copied
// by one DMA transfer.  An ordinary pageable buffer would otherwise go through
// the driver's own single-threaded staging, at a fraction of the PCIe rate, so
// it is copied here in chunks through two page-locked staging buffers owned by
// the library: host threads fill (or drain) one buffer while the DMA engine
// moves the other, and the device-side layout conversion runs on the device
// copy afterwards.  The staging buffers (2 x 32 MB per device used) are
// allocated on first use and kept for the life of the process; transfers on
// one device take turns on them.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#if defined(__x86_64__)
#include <emmintrin.h>
#endif

#include "capi_internal.h"

namespace klft {
namespace {

constexpr size_t kChunk = 32u << 20;

// A small persistent pool of host threads for the staging memcpys.
class CopyPool {
 public:
  static CopyPool &get() {
    static CopyPool p;
    return p;
  }
  // fn(i) for i in [0, n) on the pool threads and the caller
  void run(int n, const std::function<void(int)> &fn) {
    if (n <= 1 || workers_.empty()) {
      for (int i = 0; i < n; ++i) fn(i);
      return;
    }
    std::unique_lock<std::mutex> lk(mu_);
    fn_ = &fn;
    next_ = 0;
    n_ = n;
    done_ = 0;
    ++gen_;
    cv_.notify_all();
    lk.unlock();
    work();
    lk.lock();
    done_cv_.wait(lk, [&] { return done_ == n_; });
    fn_ = nullptr;
  }
  int threads() const { return (int)workers_.size() + 1; }

 private:
  CopyPool() {
    unsigned hw = std::thread::hardware_concurrency();
    const int nt = (int)std::min<unsigned>(hw > 1 ? hw - 1 : 0, 15u);
    for (int i = 0; i < nt; ++i) workers_.emplace_back([this] { loop(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto &t : workers_) t.join();
  }
  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
      if (stop_) return;
      seen = gen_;
      lk.unlock();
      work();
    }
  }
  void work() {
    for (;;) {
      int i;
      const std::function<void(int)> *fn;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (!fn_ || next_ >= n_) return;
        i = next_++;
        fn = fn_;
      }
      (*fn)(i);
      std::lock_guard<std::mutex> lk(mu_);
      if (++done_ == n_) done_cv_.notify_all();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)> *fn_ = nullptr;
  int next_ = 0, n_ = 0, done_ = 0;
  unsigned long long gen_ = 0;
  bool stop_ = false;
};

// memcpy of n bytes split over the pool's threads
void par_memcpy(void *dst, const void *src, size_t n) {
  CopyPool &pool = CopyPool::get();
  const int parts = (int)std::min<size_t>((size_t)pool.threads(), std::max<size_t>(1, n >> 20));
  const size_t per = (n + parts - 1) / parts;
  pool.run(parts, [&](int i) {
    const size_t a = (size_t)i * per;
    if (a < n) memcpy((char *)dst + a, (const char *)src + a, std::min(per, n - a));
  });
}

// per device: the events belong to the device that created them
constexpr int kMaxDevices = 64;
struct Staging {
  std::mutex mu;
  void *buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
};
Staging g_staging[kMaxDevices];

bool is_pinned(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

// the current device's staging buffers (allocated on first use), or null
Staging *staging_ready(cudaError_t &e) {
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return nullptr;
  if (dev < 0 || dev >= kMaxDevices) {
    e = cudaErrorInvalidDevice;
    return nullptr;
  }
  Staging &st = g_staging[dev];
  st.mu.lock();
  if (!st.buf[0] || !st.buf[1] || !st.ev[0] || !st.ev[1]) {
    for (int k = 0; k < 2; ++k) {
      if (!st.buf[k] && (e = cudaHostAlloc(&st.buf[k], kChunk, cudaHostAllocDefault)) != cudaSuccess) break;
      if (!st.ev[k] && (e = cudaEventCreateWithFlags(&st.ev[k], cudaEventDisableTiming)) != cudaSuccess) break;
    }
    if (e != cudaSuccess) {
      st.mu.unlock();
      return nullptr;
    }
  }
  return &st;  // locked; the caller unlocks
}

// [l0, l1) of n items split over the pool's threads, at least 4096 items each
void par_range(size_t n, const std::function<void(size_t, size_t)> &fn) {
  CopyPool &pool = CopyPool::get();
  const int parts = (int)std::min<size_t>((size_t)pool.threads(), std::max<size_t>(1, n >> 12));
  const size_t per = (n + parts - 1) / parts;
  pool.run(parts, [&](int i) {
    const size_t a = (size_t)i * per;
    if (a < n) fn(a, std::min(n, a + per));
  });
}

// Per link: F stored FP32 reals on the device, D = 2 N^2 interchange doubles.
template <int NC> struct LinkReals {
  static constexpr int F = NC == 3 ? 12 : (NC == 2 ? 4 : 2);
  static constexpr int D = 2 * NC * NC;
};

// Links [l0, l1): the first F of the D doubles of each link, rounded to float
// (round to nearest, as the device's conversion), into the page-locked staging
// buffer with streaming stores (the DMA engine reads them next, not the CPU).
template <int NC>
void pack_links(float *dst, const double *src, size_t l0, size_t l1) {
  constexpr int F = LinkReals<NC>::F, D = LinkReals<NC>::D;
  for (size_t l = l0; l < l1; ++l) {
    const double *a = src + l * D;
    float *b = dst + (l - l0) * F;
#if defined(__x86_64__)
    if constexpr (F % 4 == 0) {
#pragma unroll
      for (int k = 0; k < F; k += 4) {
        const __m128 lo = _mm_cvtpd_ps(_mm_loadu_pd(a + k)), hi = _mm_cvtpd_ps(_mm_loadu_pd(a + k + 2));
        _mm_stream_ps(b + k, _mm_movelh_ps(lo, hi));
      }
    } else {
      for (int k = 0; k < F; ++k) b[k] = (float)a[k];
    }
#else
    for (int k = 0; k < F; ++k) b[k] = (float)a[k];
#endif
  }
#if defined(__x86_64__)
  _mm_sfence();
#endif
}

// Links [l0, l1) from their stored FP32 reals to the D interchange doubles:
// SU(3) row 2 = conj(row0 x row1) and SU(2) row 1 = (-conj(b), conj(a)), the
// completions the device applies when it loads a link, formed here in FP64
// (products of FP32 values are exact in FP64).  Streaming stores into a
// 16-byte aligned destination (no read of the caller's lines before writing).
template <int NC>
void unpack_links(double *dst, const float *src, size_t l0, size_t l1) {
  constexpr int F = LinkReals<NC>::F, D = LinkReals<NC>::D;
  const bool nt = ((uintptr_t)dst & 15u) == 0;
  for (size_t l = l0; l < l1; ++l) {
    const float *a = src + (l - l0) * F;
    double v[D];
#pragma unroll
    for (int k = 0; k < F; ++k) v[k] = (double)a[k];
    if constexpr (NC == 3) {
      // m2j = conj(m0k m1q - m0q m1k), (j, k, q) = (0, 1, 2), (1, 2, 0), (2, 0, 1)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int k = (j + 1) % 3, q = (j + 2) % 3;
        const double ar = v[2 * k], ai = v[2 * k + 1], br = v[6 + 2 * q], bi = v[6 + 2 * q + 1];
        const double cr = v[2 * q], ci = v[2 * q + 1], dr = v[6 + 2 * k], di = v[6 + 2 * k + 1];
        v[12 + 2 * j] = (ar * br - ai * bi) - (cr * dr - ci * di);
        v[12 + 2 * j + 1] = -((ar * bi + ai * br) - (cr * di + ci * dr));
      }
    } else if constexpr (NC == 2) {
      v[4] = -v[2];
      v[5] = v[3];
      v[6] = v[0];
      v[7] = -v[1];
    }
    double *b = dst + l * D;
#if defined(__x86_64__)
    if (nt) {
#pragma unroll
      for (int k = 0; k < D; k += 2) _mm_stream_pd(b + k, _mm_loadu_pd(v + k));
      continue;
    }
#endif
    std::memcpy(b, v, sizeof v);
  }
#if defined(__x86_64__)
  _mm_sfence();
#endif
}

template <typename F> void by_nc(int nc, F &&f) {
  if (nc == 3) f(std::integral_constant<int, 3>());
  else if (nc == 2) f(std::integral_constant<int, 2>());
  else f(std::integral_constant<int, 1>());
}

}  // namespace

cudaError_t upload_links_f32(void *dst, const double *src, size_t nlinks, int nc, cudaStream_t st) {
  const int fr = nc == 3 ? 12 : (nc == 2 ? 4 : 2);
  cudaError_t e = cudaSuccess;
  Staging *sg = staging_ready(e);
  if (!sg) return e;
  std::lock_guard<std::mutex> lk(sg->mu, std::adopt_lock);
  const size_t per_chunk = kChunk / (fr * sizeof(float));
  for (size_t k = 0, l0 = 0; l0 < nlinks; ++k, l0 += per_chunk) {
    const int b = (int)(k & 1);
    const size_t n = std::min(per_chunk, nlinks - l0);
    if ((e = cudaEventSynchronize(sg->ev[b])) != cudaSuccess) return e;
    float *stage = (float *)sg->buf[b];
    by_nc(nc, [&](auto ncv) {
      constexpr int NC = decltype(ncv)::value;
      par_range(n, [&](size_t a, size_t z) { pack_links<NC>(stage + a * fr, src, l0 + a, l0 + z); });
    });
    if ((e = cudaMemcpyAsync((float *)dst + l0 * fr, stage, n * fr * sizeof(float), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
      return e;
    if ((e = cudaEventRecord(sg->ev[b], st)) != cudaSuccess) return e;
  }
  for (int b = 0; b < 2; ++b)
    if ((e = cudaEventSynchronize(sg->ev[b])) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t download_links_f32(double *dst, const void *src, size_t nlinks, int nc, cudaStream_t st) {
  const int fr = nc == 3 ? 12 : (nc == 2 ? 4 : 2);
  cudaError_t e = cudaSuccess;
  Staging *sg = staging_ready(e);
  if (!sg) return e;
  std::lock_guard<std::mutex> lk(sg->mu, std::adopt_lock);
  const size_t per_chunk = kChunk / (fr * sizeof(float));
  const size_t nchunks = (nlinks + per_chunk - 1) / per_chunk;
  // chunk k goes to buffer k & 1 and is expanded into the caller's array once
  // its copy is done, while the next chunk's copy runs
  for (size_t k = 0; k < nchunks + 1; ++k) {
    if (k < nchunks) {
      const int b = (int)(k & 1);
      const size_t l0 = k * per_chunk, n = std::min(per_chunk, nlinks - l0);
      if ((e = cudaMemcpyAsync(sg->buf[b], (const float *)src + l0 * fr, n * fr * sizeof(float),
                               cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
      if ((e = cudaEventRecord(sg->ev[b], st)) != cudaSuccess) return e;
    }
    if (k >= 1) {
      const size_t j = k - 1;
      const int b = (int)(j & 1);
      const size_t l0 = j * per_chunk, n = std::min(per_chunk, nlinks - l0);
      if ((e = cudaEventSynchronize(sg->ev[b])) != cudaSuccess) return e;
      const float *stage = (const float *)sg->buf[b];
      by_nc(nc, [&](auto ncv) {
        constexpr int NC = decltype(ncv)::value;
        par_range(n, [&](size_t a, size_t z) { unpack_links<NC>(dst, stage + a * fr, l0 + a, l0 + z); });
      });
    }
  }
  return cudaSuccess;
}

cudaError_t copy_host_to_device(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (is_pinned(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  cudaError_t e = cudaSuccess;
  Staging *sg = staging_ready(e);
  if (!sg) return e;
  std::lock_guard<std::mutex> lk(sg->mu, std::adopt_lock);
  size_t off = 0;
  for (int k = 0; off < bytes; ++k) {
    const int b = k & 1;
    const size_t n = std::min(kChunk, bytes - off);
    // the buffer's previous transfer must have left it before it is refilled
    if ((e = cudaEventSynchronize(sg->ev[b])) != cudaSuccess) return e;
    par_memcpy(sg->buf[b], (const char *)src + off, n);
    if ((e = cudaMemcpyAsync((char *)dst + off, sg->buf[b], n, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(sg->ev[b], st)) != cudaSuccess) return e;
    off += n;
  }
  // the staging buffers are shared by all lattices of the device: drain before returning
  for (int b = 0; b < 2; ++b)
    if ((e = cudaEventSynchronize(sg->ev[b])) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t copy_device_to_host(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (is_pinned(dst)) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
    return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
  }
  cudaError_t e = cudaSuccess;
  Staging *sg = staging_ready(e);
  if (!sg) return e;
  std::lock_guard<std::mutex> lk(sg->mu, std::adopt_lock);
  const size_t nchunks = (bytes + kChunk - 1) / kChunk;
  // chunk k goes to buffer k & 1; it is drained to the caller once its copy is
  // done, while the next chunk's copy runs
  for (size_t k = 0; k < nchunks + 1; ++k) {
    if (k < nchunks) {
      const int b = (int)(k & 1);
      const size_t off = k * kChunk, n = std::min(kChunk, bytes - off);
      if ((e = cudaMemcpyAsync(sg->buf[b], (const char *)src + off, n, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
      if ((e = cudaEventRecord(sg->ev[b], st)) != cudaSuccess) return e;
    }
    if (k >= 1) {
      const size_t j = k - 1;
      const int b = (int)(j & 1);
      const size_t off = j * kChunk, n = std::min(kChunk, bytes - off);
      if ((e = cudaEventSynchronize(sg->ev[b])) != cudaSuccess) return e;
      par_memcpy((char *)dst + off, sg->buf[b], n);
    }
  }
  return cudaSuccess;
}

}  // namespace klft
