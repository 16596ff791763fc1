// The CFL time step of a caller's device-resident Euler state, without any
// allocation.
//
// Some callers cannot call cudaMalloc: an application whose device memory is
// owned by its own pool allocator (every byte accounted for up front), or a
// latency-critical loop that cannot accept cudaMalloc's implicit device-wide
// synchronization.  wasl_cfl_dt_static serves them: the caller passes the
// state and receives dt in device memory it already owns, and the reduction's
// per-block partials live in g_cfl_scratch below, a fixed array that every
// GPU loading this library holds until the process exits.
//
// Limits and sharing:
//   * at most kMaxElements elements per call (larger inputs are rejected);
//   * every call on a device uses the same array: two calls whose kernels
//     overlap on that GPU (different streams, or different host threads)
//     race and may return each other's results;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.
#include <array>
#include <atomic>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "../../include/wasl_b200.h"
#include "euler_device.cuh"

namespace wasl_b200 {
namespace {

constexpr int kBlock = 256;
constexpr int kPerThread = 8;                            // elements per thread
constexpr int kMaxBlocks = 16384;                        // partials held
constexpr long long kSpan = static_cast<long long>(kBlock) * kPerThread;
constexpr long long kMaxElements = kSpan * kMaxBlocks;   // 33,554,432 elements

struct CflScratch {
  double speed[kMaxBlocks];   // largest |u|+c of each block's element range
  unsigned long long error;   // first non-physical element, code in the top byte
};

} // namespace

// 16384 x 8 B + 8 B = 128 KiB per device.
static __device__ __align__(256) CflScratch g_cfl_scratch;

namespace {

__global__ void __launch_bounds__(kBlock)
    cfl_static_partial(const double *__restrict__ state, long long ne, int M, int dimensions,
                       double gamma, CflScratch *scratch) {
  __shared__ double block_best[kBlock / 32];
  const double scale = 1.0 / sqrt(2.0);
  const long long plane = static_cast<long long>(M) * ne;
  const long long begin = static_cast<long long>(blockIdx.x) * kSpan;
  double best = 0.0;
  for (int k = 0; k < kPerThread; ++k) {
    const long long e = begin + static_cast<long long>(k) * kBlock + threadIdx.x;
    if (e >= ne)
      break;
    const double s[4] = {scale * state[e], scale * state[plane + e], scale * state[2 * plane + e],
                         scale * state[3 * plane + e]};
    const Prim<double> v = primitive(gamma, s);
    if (!(s[0] > 0.0 && v.p > 0.0)) {
      raise_error(&scratch->error, kNonPhysicalAverage, e);
      continue;
    }
    const double velocity = dimensions == 1 ? fabs(v.vx) : hypot(v.vx, v.vy);
    best = smax(best, velocity + sound_speed(gamma, v));
  }
  for (int off = 16; off > 0; off >>= 1)
    best = smax(best, __shfl_down_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0)
    block_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = block_best[0];
    for (int w = 1; w < kBlock / 32; ++w)
      b = smax(b, block_best[w]);
    scratch->speed[blockIdx.x] = b;
  }
}

__global__ void __launch_bounds__(kBlock)
    cfl_static_final(const CflScratch *scratch, int blocks, double cfl, double length, int p,
                     double *dt) {
  __shared__ double block_best[kBlock / 32];
  double best = 0.0;
  for (int b = threadIdx.x; b < blocks; b += kBlock)
    best = smax(best, scratch->speed[b]);
  for (int off = 16; off > 0; off >>= 1)
    best = smax(best, __shfl_down_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0)
    block_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    double speed = block_best[0];
    for (int w = 1; w < kBlock / 32; ++w)
      speed = smax(speed, block_best[w]);
    *dt = speed > 0.0 ? cfl * length / (speed * (2 * p + 1)) : 0.0;
  }
}

// Device address of g_cfl_scratch, looked up once per device.
std::array<std::atomic<CflScratch *>, 64> scratch_of_device{};

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
                "cfl: element count " + std::to_string(element_count) +
                    " outside 1.." + std::to_string(kMaxElements) +
                    " (the static scratch holds " + std::to_string(kMaxBlocks) +
                    " block partials)");
  if (mode_count < 1 || (dimensions != 1 && dimensions != 2) || polynomial_order < 0)
    return fail(error, error_length, WASL_ERR_ARGUMENT, "cfl: invalid modes or dimensions");
  int device = 0;
  cudaError_t rc = cudaGetDevice(&device);
  if (rc != cudaSuccess || device < 0 || device >= static_cast<int>(scratch_of_device.size()))
    return fail(error, error_length, WASL_ERR_CUDA, "cfl: no usable CUDA device");
  CflScratch *scratch = scratch_of_device[device].load();
  if (!scratch) {
    void *address = nullptr;
    rc = cudaGetSymbolAddress(&address, g_cfl_scratch);
    if (rc != cudaSuccess)
      return fail(error, error_length, WASL_ERR_CUDA,
                  std::string("cfl: scratch address: ") + cudaGetErrorString(rc));
    scratch = static_cast<CflScratch *>(address);
    scratch_of_device[device].store(scratch);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The error word must start at zero; the partials are fully overwritten.
  rc = cudaMemsetAsync(&scratch->error, 0, sizeof(unsigned long long), s);
  const int blocks = static_cast<int>((element_count + kSpan - 1) / kSpan);
  if (rc == cudaSuccess) {
    cfl_static_partial<<<blocks, kBlock, 0, s>>>(state, element_count, mode_count, dimensions,
                                                 gamma, scratch);
    cfl_static_final<<<1, kBlock, 0, s>>>(scratch, blocks, cfl, length, polynomial_order, dt);
    rc = cudaGetLastError();
  }
  unsigned long long word = 0;
  if (rc == cudaSuccess)
    rc = cudaMemcpyAsync(&word, &scratch->error, sizeof(word), cudaMemcpyDeviceToHost, s);
  if (rc == cudaSuccess)
    rc = cudaStreamSynchronize(s);
  if (rc != cudaSuccess)
    return fail(error, error_length, WASL_ERR_CUDA, std::string("cfl: ") + cudaGetErrorString(rc));
  if (word)
    return fail(error, error_length, WASL_ERR_NONPHYSICAL,
                "simulation: Euler cell average is not physical (element " +
                    std::to_string(word & 0xffffffffffffffULL) + ")");
  return WASL_OK;
}
