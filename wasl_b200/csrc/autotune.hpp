// Launch-shape autotuner: times each variant of a kernel on the caller's
// stream with CUDA events and keeps the fastest, per key (kernel, device,
// polynomial order, rule order and problem-size class), for the rest of the
// process.  Variants must be side-effect free with respect to the state they
// are timed on (the callers run a stage into scratch buffers).
#pragma once

#include <functional>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace wasl_b200 {

struct TuneResult {
  int choice = -1;
  std::vector<double> ms; // mean time per run of each variant
};

// run(i) enqueues variant i once on `stream`.  Each variant runs once
// untimed, then `reps` times between two events; the smallest mean wins.
TuneResult autotune(const std::string &key, int variants, const std::function<void(int)> &run,
                    cudaStream_t stream, int reps = 5);

// The size class of a problem of n elements (its binary order of magnitude),
// for tuning keys.
int size_class(long long n);

} // namespace wasl_b200
