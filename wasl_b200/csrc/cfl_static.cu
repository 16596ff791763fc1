// The CFL time step of a caller's device-resident Euler state, without any
// allocation.
//
// Some callers cannot call cudaMalloc: an application whose device memory is
// owned by its own pool allocator (every byte accounted for up front), or a
// latency-critical loop that cannot accept cudaMalloc's implicit device-wide
// synchronization.  wasl_cfl_dt_static serves them: the caller passes the
// state and receives dt in device memory it already owns, and the reduction's
// scratch (one (speed, element) pair per block of the fixed reduction grid,
// the block counter, the winner's record and the error word) lives in
// g_cfl_scratch below, a fixed 9.6 KiB array that every GPU loading this
// library holds until the process exits.
//
// The rule is the solver handle's, step for step: the one-pass reduction
// kernel of the handles (launch_cfl) finds the largest cell-average wave
// speed and the smallest element reaching it, and the host re-evaluates that
// element's speed with the C library's functions (host_cell_speed) and forms
// dt = cfl length / (speed (2p + 1)).  So the dt is the one
// wasl_gpu_stable_dt returns for the same state, bit for bit.
//
// Limits and sharing:
//   * at most kMaxElements elements per call (larger inputs are rejected);
//   * every call on a device uses the same array: two calls whose kernels
//     overlap on that GPU (different streams, or different host threads)
//     race and may return each other's results;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current;
//   * every call copies the winner back to the host and synchronizes the
//     stream, so no call can be made while that stream is being captured.
#include <array>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "../../include/wasl_b200.h"
#include "kernels.hpp"
#include "solver.hpp"

namespace wasl_b200 {
namespace {

// Element indices of the library's meshes are 32-bit.
constexpr long long kMaxElements = 2147483647LL;
// The reduction's words (kCflResultWords) and, after them, the error word.
constexpr std::size_t kScratchWords = kCflResultWords + 1;

} // namespace

static __device__ __align__(256) unsigned long long g_cfl_scratch[kScratchWords];

namespace {

// Device address of g_cfl_scratch, looked up once per device.
std::array<std::atomic<unsigned long long *>, 64> scratch_of_device{};

int fail(char *error, size_t length, int status, const std::string &message) {
  if (error && length) {
    std::strncpy(error, message.c_str(), length - 1);
    error[length - 1] = '\0';
  }
  return status;
}

} // namespace
} // namespace wasl_b200

extern "C" int wasl_cfl_dt_static(const double *state, int64_t element_count, int mode_count,
                                  int dimensions, int polynomial_order, double gamma, double cfl,
                                  double length, double *dt, void *stream, char *error,
                                  size_t error_length) {
  using namespace wasl_b200;
  if (!state || !dt)
    return fail(error, error_length, WASL_ERR_ARGUMENT, "cfl: null state or dt pointer");
  if (element_count < 1 || element_count > kMaxElements)
    return fail(error, error_length, WASL_ERR_ARGUMENT,
                "cfl: element count " + std::to_string(element_count) + " outside 1.." +
                    std::to_string(kMaxElements) + " (32-bit element indices)");
  if (mode_count < 1 || (dimensions != 1 && dimensions != 2) || polynomial_order < 0)
    return fail(error, error_length, WASL_ERR_ARGUMENT, "cfl: invalid modes or dimensions");
  int device = 0;
  cudaError_t rc = cudaGetDevice(&device);
  if (rc != cudaSuccess || device < 0 || device >= static_cast<int>(scratch_of_device.size()))
    return fail(error, error_length, WASL_ERR_CUDA, "cfl: no usable CUDA device");
  unsigned long long *scratch = scratch_of_device[device].load();
  if (!scratch) {
    void *address = nullptr;
    rc = cudaGetSymbolAddress(&address, g_cfl_scratch);
    if (rc != cudaSuccess)
      return fail(error, error_length, WASL_ERR_CUDA,
                  std::string("cfl: scratch address: ") + cudaGetErrorString(rc));
    scratch = static_cast<unsigned long long *>(address);
    scratch_of_device[device].store(scratch);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CflArgs a;
  a.ne = element_count;
  a.M = mode_count;
  a.dimensions = dimensions;
  a.state = state;
  a.gamma = gamma;
  a.cfl = cfl;
  a.length = length;
  a.p = polynomial_order;
  a.result = scratch;
  a.dt = nullptr; // the host forms dt, as the handles do
  a.error = scratch + kCflResultWords;
  // The error word must start at zero; launch_cfl clears its own counters
  // and the pairs are fully overwritten.
  rc = cudaMemsetAsync(a.error, 0, sizeof(unsigned long long), s);
  if (rc == cudaSuccess) {
    try {
      launch_cfl(a, s);
    } catch (const std::exception &e) {
      return fail(error, error_length, WASL_ERR_CUDA, std::string("cfl: ") + e.what());
    }
    rc = cudaGetLastError();
  }
  unsigned long long words[8] = {}, word = 0;
  if (rc == cudaSuccess)
    rc = cudaMemcpyAsync(words, scratch, sizeof(words), cudaMemcpyDeviceToHost, s);
  if (rc == cudaSuccess)
    rc = cudaMemcpyAsync(&word, a.error, sizeof(word), cudaMemcpyDeviceToHost, s);
  if (rc == cudaSuccess)
    rc = cudaStreamSynchronize(s);
  if (rc != cudaSuccess)
    return fail(error, error_length, WASL_ERR_CUDA, std::string("cfl: ") + cudaGetErrorString(rc));
  if (word)
    return fail(error, error_length, WASL_ERR_NONPHYSICAL,
                "simulation: Euler cell average is not physical (element " +
                    std::to_string(word & 0xffffffffffffffULL) + ")");
  double mode0[4];
  for (int v = 0; v < 4; ++v)
    mode0[v] = bits_to_double(words[2 + v]);
  const double speed = host_cell_speed(gamma, mode0, dimensions);
  const double value = speed > 0.0 ? cfl * length / (speed * (2 * polynomial_order + 1)) : 0.0;
  rc = cudaMemcpyAsync(dt, &value, sizeof(value), cudaMemcpyHostToDevice, s);
  if (rc == cudaSuccess)
    rc = cudaStreamSynchronize(s);
  if (rc != cudaSuccess)
    return fail(error, error_length, WASL_ERR_CUDA, std::string("cfl: ") + cudaGetErrorString(rc));
  return WASL_OK;
}
