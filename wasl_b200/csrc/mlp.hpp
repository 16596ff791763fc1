// The learned troubled-cell indicator (mlp.cu): shapes, kernel launchers and
// the trainer behind wasl_mlp_*.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "solver.hpp"

namespace wasl_b200 {

constexpr int kMlpHidden = 64;
constexpr int kMlpMaxFeatures = 48;
constexpr int kMlpMaxModes = 10; // P3 triangles
constexpr int kMlpBatch = 64; // samples per training block

// Offsets of each parameter block in the flat FP32 vector:
// W1 [64][F], b1 [64], W2 [64][64], b2 [64], w3 [64], b3.
struct MlpShape {
  int features = 0;
  std::int64_t w1 = 0, b1 = 0, w2 = 0, b2 = 0, w3 = 0, b3 = 0, count = 0;
};

MlpShape mlp_shape(int features);
// Features for M modes per variable: 4 (M - 1) + 3, padded to a multiple of 16.
int mlp_features_for_modes(int M);

struct MlpIndicatorArgs {
  MlpShape shape;
  const float *params = nullptr; // FP32 master weights (rounded to BF16 in the kernel)
  float lo = 0.1f, hi = 0.9f;    // confidence band handed to the reference sensor
  const double *state = nullptr; // U[var][mode][elem]
  std::int64_t ne = 0;
  int M = 0;
  const std::int32_t *neighbors = nullptr; // limiter stencil [ne][3]
  double threshold = 1e-3;
  int highest_degree_begin = 0;
  std::uint8_t *flags = nullptr;
  std::int32_t *troubled = nullptr;
  std::int32_t *troubled_count = nullptr;
  unsigned long long *stats = nullptr; // [6], see mlp_indicator_kernel
  float *logits = nullptr;             // optional [ne]
  void *records = nullptr;             // scratch, kMlpRecordBytes x ne
  unsigned long long *error = nullptr; // the handle's error word (kMlpWaitCode)
  int kernel = 0;                      // 0 tcgen05 MMAs, 1 mma.sync
};

// Error-word code of an inference kernel whose tensor-core wait ran out.
constexpr int kMlpWaitCode = 5;

// Bytes per element of the inference's per-element records.
constexpr std::size_t kMlpRecordBytes = 32;

void launch_mlp_features(const double *state, std::int64_t ne, int M,
                         const std::int32_t *neighbors, int F, double threshold,
                         int highest_degree_begin, float *features, std::uint8_t *labels,
                         cudaStream_t stream);
void launch_mlp_train(const MlpShape &shape, const float *params, const float *features,
                      const std::uint8_t *labels, std::int64_t n, std::int64_t first,
                      std::int64_t blocks, float pos_weight, float *grad, double *loss,
                      cudaStream_t stream);
void launch_mlp_adam(std::int64_t count, float *params, float *grad, float *m1, float *m2,
                     float lr, float beta1, float beta2, float eps, std::int64_t step, float scale,
                     cudaStream_t stream);
void launch_mlp_predict(const MlpShape &shape, const float *params, const float *features,
                        std::int64_t n, float *logits, cudaStream_t stream);
void launch_mlp_indicator(const MlpIndicatorArgs &args, cudaStream_t stream);

// Device-resident network, training data and Adam state.
class MlpTrainer {
public:
  MlpTrainer(int features, std::uint64_t seed, int device);
  ~MlpTrainer();
  MlpTrainer(const MlpTrainer &) = delete;
  MlpTrainer &operator=(const MlpTrainer &) = delete;
  const MlpShape &shape() const { return shape_; }
  void set_data(const float *features, const std::uint8_t *labels, std::int64_t n);
  // `steps` Adam steps on mini-batches of `batch` samples (a multiple of the
  // block batch), cycling through the data in order; the mean loss of the
  // last step.
  double train(std::int64_t steps, std::int64_t batch, double lr, double pos_weight);
  // The gradient of the mean weighted loss over the given samples at the
  // current weights, and that loss.
  double gradient(const float *features, const std::uint8_t *labels, std::int64_t n,
                  double pos_weight, float *grad_out);
  void predict(const float *features, std::int64_t n, float *logits);
  void get(float *params) const;
  void set(const float *params);
  cudaStream_t stream() const { return stream_; }

private:
  MlpShape shape_;
  cudaStream_t stream_ = nullptr;
  DeviceArray<float> params_, grad_, m1_, m2_, data_;
  DeviceArray<std::uint8_t> labels_;
  DeviceArray<double> loss_;
  std::int64_t n_ = 0, cursor_ = 0, step_ = 0;
};

} // namespace wasl_b200
