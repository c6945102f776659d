// tuner.cu -- launch-shape tuner, the counterpart of klft's MDRange tile tuner
// (Tuner.hpp:73-358).
//
// With tuning enabled (KLFT_TUNING=1 in the reference's env convention), the
// first launch of a kernel under a given key times each candidate launch shape
// (block size or CTAs per SM; min over a few CUDA-event-timed runs, like the
// reference's min over STREAM_NTIMES runs) and keeps the fastest; later
// launches reuse it.  Keys follow the reference:
//   "<id>_rank_<r>_start_<0_..._>end_<e0_..._e{r-1}_>"
// and the cache file (KLFT_CACHE_FILE) uses its text format, one line per key:
//   "<rank> <key> <v0> ... <v{r-1}>"
// where v0 is the tuned launch parameter (the remaining entries are 1).
// Results of every kernel are independent of the launch shape (per-site random
// streams, fixed-order reductions), so tuning changes speed only.  Kernels that
// update the links are timed on a scratch copy, so tuning never perturbs a chain.
#include <cstdio>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/klft_b200.h"
#include "capi_internal.h"
#include "tuner.h"

namespace klft {

namespace {
struct TunerState {
  int enabled = 0;
  int verbosity = 0;
  std::mutex mtx;
  std::map<std::string, std::vector<int>> table;
};
TunerState &state() {
  static TunerState s;
  return s;
}
}  // namespace

std::string tune_key(const std::string &id, int rank, const int *end) {
  std::string s = id + "_rank_" + std::to_string(rank) + "_start_";
  for (int i = 0; i < rank; ++i) s += "0_";
  s += "end_";
  for (int i = 0; i < rank; ++i) s += std::to_string(end[i]) + "_";
  return s;
}

bool tuner_enabled() { return state().enabled != 0; }

int tuned_param(const std::string &key, int rank, const std::vector<int> &candidates, int fallback,
                const std::function<float(int)> &time_candidate, bool may_tune) {
  TunerState &st = state();
  if (!st.enabled) return fallback;
  {
    std::lock_guard<std::mutex> g(st.mtx);
    auto it = st.table.find(key);
    if (it != st.table.end() && !it->second.empty()) {
      if (st.verbosity > 2) printf("Tuning found for kernel %s, launch parameter: %d\n", key.c_str(), it->second[0]);
      return it->second[0];
    }
  }
  if (!may_tune || candidates.empty()) return fallback;
  if (st.verbosity > 2) printf("Start tuning for kernel %s\n", key.c_str());
  int best = fallback;
  float best_ms = 3.4e38f;
  for (int c : candidates) {
    const float ms = time_candidate(c);
    if (st.verbosity > 2) printf("Current launch parameter: %d, time: %11.4e s\n", c, ms * 1e-3);
    if (ms >= 0.f && ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  if (st.verbosity > 2) {
    printf("Best launch parameter: %d\n", best);
    printf("Best Time: %11.4e s\n", best_ms * 1e-3);
  }
  std::vector<int> v(rank > 0 ? rank : 1, 1);
  v[0] = best;
  std::lock_guard<std::mutex> g(st.mtx);
  st.table[key] = v;
  return best;
}

float time_launches(cudaStream_t stream, int reps, const std::function<cudaError_t()> &launch) {
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess) return -1.f;
  if (cudaEventCreate(&b) != cudaSuccess) {
    cudaEventDestroy(a);
    return -1.f;
  }
  float best = -1.f;
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(a, stream);
    if (launch() != cudaSuccess) {
      best = -1.f;
      break;
    }
    cudaEventRecord(b, stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (r > 0 && (best < 0.f || ms < best)) best = ms;  // the first run warms up
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

}  // namespace klft

using namespace klft;

extern "C" {

klft_status klft_tuner_configure(int enabled, int verbosity) {
  TunerState &st = state();
  std::lock_guard<std::mutex> g(st.mtx);
  st.enabled = enabled;
  st.verbosity = verbosity;
  return KLFT_OK;
}

// Tuner.hpp:268-302 writeTuneCache
klft_status klft_tuner_write_cache(const char *path) {
  if (!path) return fail(KLFT_EINVAL, "klft_tuner_write_cache: null path");
  TunerState &st = state();
  std::ofstream f(path, std::ios::out);
  if (!f.is_open()) return fail(KLFT_EINVAL, "Error: could not open cache file %s", path);
  std::lock_guard<std::mutex> g(st.mtx);
  for (const auto &e : st.table) {
    f << e.second.size() << " " << e.first << " ";
    for (int v : e.second) f << v << " ";
    f << "\n";
  }
  if (st.verbosity > 0) printf("Tuning hash table written to %s\n", path);
  return KLFT_OK;
}

// Tuner.hpp:305-358 readTuneCache
klft_status klft_tuner_read_cache(const char *path) {
  if (!path) return fail(KLFT_EINVAL, "klft_tuner_read_cache: null path");
  TunerState &st = state();
  std::ifstream f(path);
  if (!f.is_open()) {
    printf("Could not open cache file %s\n", path);
    return fail(KLFT_EINVAL, "could not open cache file %s", path);
  }
  std::string line;
  std::lock_guard<std::mutex> g(st.mtx);
  while (std::getline(f, line)) {
    std::istringstream iss(line);
    int rank = 0;
    std::string key;
    if (!(iss >> rank)) continue;
    if (rank < 1 || rank > 4) {
      printf("Error: unsupported rank %d\n", rank);
      continue;
    }
    iss >> key;
    std::vector<int> v(rank, 1);
    for (int i = 0; i < rank; ++i) iss >> v[i];
    st.table[key] = v;
  }
  if (st.verbosity > 0) printf("Tuning hash table read from %s\n", path);
  return KLFT_OK;
}

klft_status klft_tuner_lookup(const char *key, int *values, int *rank) {
  if (!key) return fail(KLFT_EINVAL, "klft_tuner_lookup: null key");
  TunerState &st = state();
  std::lock_guard<std::mutex> g(st.mtx);
  auto it = st.table.find(key);
  if (it == st.table.end()) {
    if (rank) *rank = 0;
    return KLFT_OK;
  }
  if (rank) *rank = (int)it->second.size();
  if (values)
    for (size_t i = 0; i < it->second.size(); ++i) values[i] = it->second[i];
  return KLFT_OK;
}

klft_status klft_tuner_clear(void) {
  TunerState &st = state();
  std::lock_guard<std::mutex> g(st.mtx);
  st.table.clear();
  return KLFT_OK;
}

}  // extern "C"
