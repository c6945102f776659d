// checkpoint.cu -- gauge configuration checkpoints.
//
// The reference has no configuration I/O at all (measurements stay in host
// vectors until the end of a run, GaugeObservable.hpp:40-44).  Because every
// random number here is a function of (seed, chain, counters, site), a
// checkpoint of the links, the stream and the counters is a complete resume
// point: a run restored from it continues bit for bit.
//
// File layout (little-endian, 128-byte header, then the payload):
//   0  char[8]  "KLFTCKPT"
//   8  u32      format version (1)
//  12  u32      header bytes (128)
//  16  i32      Nc, ndims, L[4], precision          (7 x 4 B)
//  44  i32      defect active, len, pos[3]          (5 x 4 B)
//  64  u64      seed, chain
//  80  u32      counters[3] (sweep, trajectory, cycle)
//  92  u32      open-boundary direction + 1 (0: periodic)
//  96  f64      defect coefficient
// 104  u64      payload bytes
// 112  u64      FNV-1a 64 of the payload
// 120  u64      FNV-1a 64 of header bytes 0..119
// payload: links in the host interchange layout, complex128 (V, Nd, Nc, Nc),
// site = x0 + L0 (x1 + L1 (x2 + L2 x3)); the mixed form's FP32 values convert
// to and from double exactly.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/klft_b200.h"
#include "capi_internal.h"

using namespace klft;

namespace {

constexpr char kMagic[8] = {'K', 'L', 'F', 'T', 'C', 'K', 'P', 'T'};
constexpr uint32_t kVersion = 1, kHeader = 128;

uint64_t fnv1a(const void *p, size_t n, uint64_t h = 1469598103934665603ull) {
  const unsigned char *b = (const unsigned char *)p;
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

template <typename T>
void put(unsigned char *h, size_t off, T v) { std::memcpy(h + off, &v, sizeof v); }
template <typename T>
T get(const unsigned char *h, size_t off) {
  T v;
  std::memcpy(&v, h + off, sizeof v);
  return v;
}

struct FileCloser {
  void operator()(FILE *f) const { if (f) std::fclose(f); }
};

}  // namespace

extern "C" {

klft_status klft_checkpoint_write(klft_lattice *lat, const char *path) {
  if (!lat || !path) return fail(KLFT_EINVAL, "klft_checkpoint_write: null pointer");
  const size_t n = (size_t)lat->g.V * lat->g.nd * lat->nc * lat->nc * 2;
  std::vector<double> links(n);
  klft_status s = klft_lattice_download(lat, links.data());
  if (s != KLFT_OK) return s;
  uint32_t ctr[4];
  Defect df;
  uint64_t seed, chain;
  int open_mu;
  {
    std::lock_guard<std::mutex> g(lat->mtx);
    cudaError_t e = cudaMemcpyAsync(ctr, lat->d_counters, sizeof ctr, cudaMemcpyDeviceToHost, lat->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(lat->stream);
    if (e != cudaSuccess) return cuda_fail(e, "klft_checkpoint_write: counters");
    df = lat->defect;
    seed = lat->seed;
    chain = lat->chain;
    open_mu = lat->g.open_mu;
  }
  unsigned char h[kHeader];
  std::memset(h, 0, sizeof h);
  std::memcpy(h, kMagic, 8);
  put<uint32_t>(h, 8, kVersion);
  put<uint32_t>(h, 12, kHeader);
  put<int32_t>(h, 16, lat->nc);
  put<int32_t>(h, 20, lat->g.nd);
  for (int d = 0; d < 4; ++d) put<int32_t>(h, 24 + 4 * d, d < lat->g.nd ? lat->g.L[d] : 1);
  put<int32_t>(h, 40, lat->precision);
  put<int32_t>(h, 44, df.active);
  put<int32_t>(h, 48, df.len);
  for (int k = 0; k < 3; ++k) put<int32_t>(h, 52 + 4 * k, df.pos[k]);
  put<uint64_t>(h, 64, seed);
  put<uint64_t>(h, 72, chain);
  for (int k = 0; k < 3; ++k) put<uint32_t>(h, 80 + 4 * k, ctr[k]);
  put<uint32_t>(h, 92, (uint32_t)(open_mu + 1));
  put<double>(h, 96, df.c);
  put<uint64_t>(h, 104, (uint64_t)(n * sizeof(double)));
  put<uint64_t>(h, 112, fnv1a(links.data(), n * sizeof(double)));
  put<uint64_t>(h, 120, fnv1a(h, 120));
  // write to a temporary name and rename, so an interrupted write never leaves
  // a truncated file under the checkpoint's name
  std::string tmp = std::string(path) + ".tmp";
  {
    std::unique_ptr<FILE, FileCloser> f(std::fopen(tmp.c_str(), "wb"));
    if (!f) return fail(KLFT_EINVAL, "klft_checkpoint_write: cannot open %s", tmp.c_str());
    if (std::fwrite(h, 1, kHeader, f.get()) != kHeader ||
        std::fwrite(links.data(), sizeof(double), n, f.get()) != n || std::fflush(f.get()) != 0)
      return fail(KLFT_EINVAL, "klft_checkpoint_write: write to %s failed", tmp.c_str());
  }
  if (std::rename(tmp.c_str(), path) != 0) return fail(KLFT_EINVAL, "klft_checkpoint_write: rename to %s failed", path);
  return KLFT_OK;
}

klft_status klft_checkpoint_read(const char *path, klft_lattice **out) {
  if (!path || !out) return fail(KLFT_EINVAL, "klft_checkpoint_read: null pointer");
  *out = nullptr;
  std::unique_ptr<FILE, FileCloser> f(std::fopen(path, "rb"));
  if (!f) return fail(KLFT_EINVAL, "klft_checkpoint_read: cannot open %s", path);
  unsigned char h[kHeader];
  if (std::fread(h, 1, kHeader, f.get()) != kHeader) return fail(KLFT_EINVAL, "klft_checkpoint_read: short header");
  if (std::memcmp(h, kMagic, 8) != 0) return fail(KLFT_EINVAL, "klft_checkpoint_read: %s is not a checkpoint", path);
  if (get<uint32_t>(h, 8) != kVersion || get<uint32_t>(h, 12) != kHeader)
    return fail(KLFT_EINVAL, "klft_checkpoint_read: unsupported format version %u", get<uint32_t>(h, 8));
  if (get<uint64_t>(h, 120) != fnv1a(h, 120)) return fail(KLFT_EINVAL, "klft_checkpoint_read: header checksum mismatch");
  const int nc = get<int32_t>(h, 16), nd = get<int32_t>(h, 20), prec = get<int32_t>(h, 40);
  int L[4];
  long long V = 1;
  for (int d = 0; d < 4; ++d) L[d] = get<int32_t>(h, 24 + 4 * d);
  if (nc < 1 || nc > 3 || nd < 2 || nd > 4) return fail(KLFT_EINVAL, "klft_checkpoint_read: bad group or dims");
  if (get<uint32_t>(h, 92) > (uint32_t)nd) return fail(KLFT_EINVAL, "klft_checkpoint_read: bad open-boundary direction");
  for (int d = 0; d < nd; ++d) {
    if (L[d] < 2 || (L[d] & 1)) return fail(KLFT_EINVAL, "klft_checkpoint_read: bad extent");
    V *= L[d];
    if (V > 0x7fffffffLL) return fail(KLFT_EINVAL, "klft_checkpoint_read: bad volume");
  }
  const size_t n = (size_t)V * nd * nc * nc * 2;
  if (get<uint64_t>(h, 104) != n * sizeof(double)) return fail(KLFT_EINVAL, "klft_checkpoint_read: payload size mismatch");
  std::vector<double> links(n);
  if (std::fread(links.data(), sizeof(double), n, f.get()) != n)
    return fail(KLFT_EINVAL, "klft_checkpoint_read: truncated payload");
  if (get<uint64_t>(h, 112) != fnv1a(links.data(), n * sizeof(double)))
    return fail(KLFT_EINVAL, "klft_checkpoint_read: payload checksum mismatch");
  klft_lattice *lat = nullptr;
  klft_status s = klft_lattice_create(nc, nd, L, prec, KLFT_START_COLD, get<uint64_t>(h, 64), &lat);
  if (s != KLFT_OK) return s;
  s = klft_lattice_upload(lat, links.data());
  if (s == KLFT_OK) s = klft_lattice_set_stream(lat, get<uint64_t>(h, 64), get<uint64_t>(h, 72));
  if (s == KLFT_OK && get<int32_t>(h, 44)) {
    const int pos[3] = {get<int32_t>(h, 52), get<int32_t>(h, 56), get<int32_t>(h, 60)};
    s = klft_lattice_set_defect(lat, get<int32_t>(h, 48), pos, get<double>(h, 96));
  }
  const uint32_t open1 = get<uint32_t>(h, 92);
  if (s == KLFT_OK && open1 > 0) s = klft_lattice_set_open_boundary(lat, (int)open1 - 1);
  if (s == KLFT_OK) {
    uint32_t ctr[4] = {0, 0, 0, 0};
    for (int k = 0; k < 3; ++k) ctr[k] = get<uint32_t>(h, 80 + 4 * k);
    std::lock_guard<std::mutex> g(lat->mtx);
    cudaError_t e = cudaMemcpyAsync(lat->d_counters, ctr, sizeof ctr, cudaMemcpyHostToDevice, lat->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(lat->stream);
    if (e != cudaSuccess) s = cuda_fail(e, "klft_checkpoint_read: counters");
  }
  if (s != KLFT_OK) {
    klft_lattice_destroy(lat);
    return s;
  }
  *out = lat;
  return KLFT_OK;
}

}  // extern "C"
