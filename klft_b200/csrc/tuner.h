// tuner.h -- internal interface of the launch-shape tuner (tuner.cu).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

namespace klft {

// "<id>_rank_<r>_start_0_..._end_<e...>_" as klft's tune_and_launch_for builds it
std::string tune_key(const std::string &id, int rank, const int *end);
bool tuner_enabled();
// The tuned launch parameter for key: fallback when tuning is off; the cached
// value when present; otherwise (when may_tune) the fastest candidate, timed
// with time_candidate (milliseconds, negative = unusable).
int tuned_param(const std::string &key, int rank, const std::vector<int> &candidates, int fallback,
                const std::function<float(int)> &time_candidate, bool may_tune);
// min over reps (after one warm-up run) of CUDA-event times of launch() on stream
float time_launches(cudaStream_t stream, int reps, const std::function<cudaError_t()> &launch);

}  // namespace klft
