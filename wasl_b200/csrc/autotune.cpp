// Launch-shape autotuner (see autotune.hpp).
#include "autotune.hpp"

#include <map>
#include <mutex>
#include <stdexcept>

namespace wasl_b200 {

void cuda_check(cudaError_t rc, const char *what);

namespace {
std::mutex mutex;
std::map<std::string, TuneResult> cache;
} // namespace

int size_class(long long n) {
  int c = 0;
  while (n > 1) {
    n >>= 1;
    ++c;
  }
  return c;
}

TuneResult autotune(const std::string &key, int variants, const std::function<void(int)> &run,
                    cudaStream_t stream, int reps) {
  int device = 0;
  cuda_check(cudaGetDevice(&device), "cudaGetDevice");
  const std::string full = key + "/dev" + std::to_string(device);
  {
    std::lock_guard<std::mutex> lock(mutex);
    const auto it = cache.find(full);
    if (it != cache.end())
      return it->second;
  }
  if (variants <= 0)
    throw std::invalid_argument("autotune: no variants");
  cudaEvent_t start, stop;
  cuda_check(cudaEventCreate(&start), "event");
  cuda_check(cudaEventCreate(&stop), "event");
  TuneResult result;
  result.ms.assign(variants, 0.0);
  for (int i = 0; i < variants; ++i) {
    run(i); // untimed: first-launch costs, caches
    cuda_check(cudaEventRecord(start, stream), "event record");
    for (int r = 0; r < reps; ++r)
      run(i);
    cuda_check(cudaEventRecord(stop, stream), "event record");
    cuda_check(cudaEventSynchronize(stop), "event sync");
    float ms = 0.0f;
    cuda_check(cudaEventElapsedTime(&ms, start, stop), "elapsed");
    result.ms[i] = static_cast<double>(ms) / reps;
    if (result.choice < 0 || result.ms[i] < result.ms[result.choice])
      result.choice = i;
  }
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  std::lock_guard<std::mutex> lock(mutex);
  cache[full] = result;
  return result;
}

} // namespace wasl_b200
