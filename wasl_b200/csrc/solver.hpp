// Solver handles behind the C-ABI: device-resident state, per-mesh setup data,
// and the SSP-RK3 step orchestration.
#pragma once

#include <chrono>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/wasl_b200.h"

namespace wasl_b200 {

// An NVTX range around a C-ABI call (header-only NVTX v3: free when no
// profiler is attached; under Nsight tools each call shows as a named range
// over the kernels it enqueues).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// Wall-clock time of a solver's setup phases (enum wasl_setup_phase), in ms.
struct SetupTimes {
  double ms[WASL_SETUP_PHASES] = {};
  std::chrono::steady_clock::time_point mark;
  void start() { mark = std::chrono::steady_clock::now(); }
  // Adds the time since the last mark to `phase` and moves the mark.
  void lap(int phase) {
    const auto now = std::chrono::steady_clock::now();
    ms[phase] += std::chrono::duration<double, std::milli>(now - mark).count();
    mark = now;
  }
};

// Failure carrying a C-ABI status code.
struct SolverError : std::runtime_error {
  int status;
  SolverError(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

void cuda_check(cudaError_t rc, const char *what);

// Owning device allocation.
template <typename T> class DeviceArray {
public:
  DeviceArray() = default;
  explicit DeviceArray(std::size_t n) { resize(n); }
  DeviceArray(const DeviceArray &) = delete;
  DeviceArray &operator=(const DeviceArray &) = delete;
  DeviceArray(DeviceArray &&o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr, o.n_ = 0; }
  ~DeviceArray() {
    if (p_)
      cudaFree(p_);
  }
  void resize(std::size_t n) {
    if (p_)
      cudaFree(p_);
    p_ = nullptr;
    n_ = n;
    if (n)
      cuda_check(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)), "cudaMalloc");
  }
  void upload(const std::vector<T> &h, cudaStream_t s = nullptr) {
    resize(h.size());
    if (!h.empty())
      cuda_check(cudaMemcpyAsync(p_, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s),
                 "upload");
  }
  T *get() const { return p_; }
  std::size_t size() const { return n_; }

private:
  T *p_ = nullptr;
  std::size_t n_ = 0;
};

// Pinned host scratch for the few scalars a step exchanges with the device.
struct PinnedScratch {
  unsigned long long *words = nullptr; // [0..7] CFL result, [8] error word
  PinnedScratch() {
    cuda_check(cudaMallocHost(reinterpret_cast<void **>(&words), 16 * sizeof(unsigned long long)),
               "pinned");
  }
  ~PinnedScratch() { cudaFreeHost(words); }
  PinnedScratch(const PinnedScratch &) = delete;
  PinnedScratch &operator=(const PinnedScratch &) = delete;
};

double bits_to_double(unsigned long long bits);

// One cell-average wave speed |u| + c (hypot(u, v) + c in 2D) evaluated on the
// host with the C library's functions, as cpp/src/time/cfl_timestep.cpp:33-47
// computes it; mode0 holds the four mode-0 coefficients.
double host_cell_speed(double gamma, const double *mode0, int dimensions);

// Throws the SolverError a device error word stands for (code in the top
// byte, element index below); returns if the word is zero.
void throw_device_error(unsigned long long word);

class Solver {
public:
  virtual ~Solver();
  virtual std::int64_t elements() const = 0;
  virtual std::int64_t faces() const = 0;
  virtual int modes() const = 0;
  virtual int variables() const = 0;
  virtual void vertices(double *out) const = 0;
  virtual void set_state(const double *host) = 0;
  virtual void get_state(double *host) = 0;
  virtual double stable_dt(double cfl) = 0;
  // The two factors of stable_dt = cfl length / (speed (2p + 1)): the
  // largest cell-average wave speed (evaluated as stable_dt evaluates it)
  // and the smallest element length.  A partitioned run reduces them over
  // ranks (max, min) and forms the same dt as one solver over the whole mesh.
  virtual void cfl_parts(double &speed, double &length) {
    (void)speed;
    (void)length;
    throw SolverError(WASL_ERR_ARGUMENT, "cfl parts: only for 2D Euler");
  }
  // stable_dt's formula from the two factors (2D Euler).
  virtual double dt_from_parts(double cfl, double speed, double length) const {
    (void)cfl, (void)speed, (void)length;
    throw SolverError(WASL_ERR_ARGUMENT, "cfl parts: only for 2D Euler");
  }
  virtual void step(double dt) = 0;
  virtual void limit() = 0; // the stage limiter applied to the current state
  // Enqueues `steps` device-resident steps; returns without waiting for
  // them (device errors stay in the error word until sync()).
  virtual void advance(double cfl, std::int64_t steps) = 0;
  // Waits for the handle's stream and raises a pending device error.
  virtual void sync() {
    cuda_check(cudaStreamSynchronize(stream_), "sync");
  }
  // The serial run loop on the device, in one launch with no host round trip
  // per step (line meshes small enough for one CTA, without the limiter).
  virtual void run_resident(double cfl, double start_time, double end_time,
                            std::uint64_t max_steps, std::uint64_t &steps, double &time) {
    (void)cfl, (void)start_time, (void)end_time, (void)max_steps, (void)steps, (void)time;
    throw SolverError(WASL_ERR_ARGUMENT, "resident run: line meshes only");
  }
  virtual void flags(std::uint8_t *out) = 0;
  virtual void mass_energy(double &mass, double &energy) = 0;
  virtual double *state_device() = 0;
  // order[i]: the caller's element stored at column i of state_device().
  virtual void element_order(std::int64_t *order) const {
    for (std::int64_t e = 0; e < elements(); ++e)
      order[e] = e;
  }
  // Quadrature of rule order r on every element: physical points and weights
  // (reference weight x |det J|), packed [element][point].
  virtual int rule_points(int rule_order) const = 0;
  virtual void quadrature(int rule_order, double *x, double *y, double *w) const = 0;
  // L2 projection of point values [element][point][variable] onto the modes,
  // stored as the state (cpp/include/wasl/dg/l2_projection.hpp:36-76).
  virtual void project(int rule_order, const double *values) = 0;
  // The state evaluated at the rule's points, [element][point][variable].
  virtual void evaluate(int rule_order, double *values) = 0;
  cudaStream_t stream() const { return stream_; }
  // The learned troubled-cell indicator (2D Euler with limiting only).
  virtual void set_indicator(const float *weights, std::int64_t count, double lo, double hi) {
    (void)weights, (void)count, (void)lo, (void)hi;
    throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: 2D Euler with limiting only");
  }
  // The inference kernel of the learned indicator: 0 tcgen05, 1 mma.sync.
  virtual void set_indicator_kernel(int kernel) {
    (void)kernel;
    throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: 2D Euler with limiting only");
  }
  virtual int indicator_features() const { return 0; }
  virtual void indicator_data(float *features, std::uint8_t *labels) {
    (void)features, (void)labels;
    throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: 2D Euler with limiting only");
  }
  virtual void indicator_logits(float *logits) {
    (void)logits;
    throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: 2D Euler with limiting only");
  }
  virtual void indicator_stats(unsigned long long *stats, bool reset) {
    (void)stats, (void)reset;
    throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: 2D Euler with limiting only");
  }
  // The kernel variant in use (-1: the form has one kernel) and, when it was
  // autotuned, the timed mean of every variant (count of them in `count`).
  virtual int kernel_choice(double *ms, int capacity, int &count) {
    (void)ms;
    (void)capacity;
    count = 0;
    return -1;
  }

  // The limiter's candidate transforms [element][candidate][target][source]
  // and the periodic trace (donors [boundary face][point], basis
  // [boundary face][point][mode]) as the kernels read them, in the caller's
  // element order (2D Euler; the trace also 2D scalar advection).
  virtual void stencil_transforms(double *out, std::int64_t count) {
    (void)out, (void)count;
    throw SolverError(WASL_ERR_ARGUMENT, "stencil transforms: 2D Euler with limiting only");
  }
  virtual void periodic_trace(std::int32_t *donors, double *basis, std::int64_t points) {
    (void)donors, (void)basis, (void)points;
    throw SolverError(WASL_ERR_ARGUMENT, "periodic trace: periodic triangle meshes only");
  }
  const SetupTimes &setup_times() const { return setup_; }
  SetupTimes &setup_times() { return setup_; }

  // Kernel accounting for measurement: every launch is counted; while
  // profiling, each stage kernel is bracketed by CUDA events on the stream it
  // is launched on.
  void profile_begin();
  void profile_end(double &stage_ms, std::int64_t &stage_kernels, std::int64_t &launches);
  // The last profile_end's stage-kernel time split by RK stage (0, 1, 2).
  const double *profile_stage_ms() const { return stage_split_; }

protected:
  void count_launches(std::int64_t n) { launches_ += n; }
  void stage_begin();
  void stage_end();

  cudaStream_t stream_ = nullptr;
  SetupTimes setup_;

private:
  bool profiling_ = false;
  std::int64_t launches_ = 0;
  std::vector<cudaEvent_t> events_;
  std::size_t events_used_ = 0;
  double stage_split_[3] = {0.0, 0.0, 0.0};
};

struct PartBoundary;
// part: the explicit boundary of one part of a partitioned periodic mesh
// (mesh.hpp), or null.
std::unique_ptr<Solver> make_solver(const wasl_gpu_config &config, std::int64_t node_count,
                                    const std::int64_t *node_tags, const double *coordinates,
                                    std::int64_t element_count, const std::int64_t *element_nodes,
                                    const PartBoundary *part = nullptr);

} // namespace wasl_b200
