// The indicator network's trainer and its extern "C" entry points
// (declared in include/wasl_b200.h).
#include <cmath>
#include <cstring>
#include <random>
#include <stdexcept>

#include "mlp.hpp"

namespace wasl_b200 {

MlpTrainer::MlpTrainer(int features, std::uint64_t seed, int device) : shape_(mlp_shape(features)) {
  cuda_check(cudaSetDevice(device), "cudaSetDevice");
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  // He-uniform initialisation of the weights, zero biases.
  std::vector<float> p(shape_.count, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](std::int64_t offset, std::int64_t count, int fan_in) {
    std::uniform_real_distribution<float> u(-std::sqrt(6.0f / fan_in), std::sqrt(6.0f / fan_in));
    for (std::int64_t i = 0; i < count; ++i)
      p[offset + i] = u(rng);
  };
  fill(shape_.w1, kMlpHidden * shape_.features, shape_.features);
  fill(shape_.w2, kMlpHidden * kMlpHidden, kMlpHidden);
  fill(shape_.w3, kMlpHidden, kMlpHidden);
  params_.upload(p, stream_);
  std::vector<float> zero(shape_.count, 0.0f);
  grad_.upload(zero, stream_);
  m1_.upload(zero, stream_);
  m2_.upload(zero, stream_);
  loss_.resize(1);
  cuda_check(cudaStreamSynchronize(stream_), "indicator network setup");
}

MlpTrainer::~MlpTrainer() {
  if (stream_)
    cudaStreamDestroy(stream_);
}

void MlpTrainer::set_data(const float *features, const std::uint8_t *labels, std::int64_t n) {
  if (n <= 0)
    throw SolverError(WASL_ERR_ARGUMENT, "indicator training: no samples");
  data_.resize(static_cast<std::size_t>(n) * shape_.features);
  labels_.resize(n);
  cuda_check(cudaMemcpyAsync(data_.get(), features, sizeof(float) * n * shape_.features,
                             cudaMemcpyHostToDevice, stream_),
             "indicator data");
  cuda_check(cudaMemcpyAsync(labels_.get(), labels, n, cudaMemcpyHostToDevice, stream_),
             "indicator labels");
  cuda_check(cudaStreamSynchronize(stream_), "indicator data");
  n_ = n;
  cursor_ = 0;
}

double MlpTrainer::train(std::int64_t steps, std::int64_t batch, double lr, double pos_weight) {
  if (n_ == 0)
    throw SolverError(WASL_ERR_ARGUMENT, "indicator training: no data set");
  if (batch <= 0 || batch % kMlpBatch != 0)
    throw SolverError(WASL_ERR_ARGUMENT, "indicator training: batch must be a positive multiple"
                                         " of 64");
  const std::int64_t blocks = batch / kMlpBatch;
  double loss = 0.0;
  for (std::int64_t s = 0; s < steps; ++s) {
    cuda_check(cudaMemsetAsync(loss_.get(), 0, sizeof(double), stream_), "loss reset");
    launch_mlp_train(shape_, params_.get(), data_.get(), labels_.get(), n_, cursor_, blocks,
                     static_cast<float>(pos_weight), grad_.get(), loss_.get(), stream_);
    cursor_ = (cursor_ + batch) % n_;
    ++step_;
    launch_mlp_adam(shape_.count, params_.get(), grad_.get(), m1_.get(), m2_.get(),
                    static_cast<float>(lr), 0.9f, 0.999f, 1e-8f, step_,
                    1.0f / static_cast<float>(batch), stream_);
  }
  cuda_check(cudaMemcpyAsync(&loss, loss_.get(), sizeof(double), cudaMemcpyDeviceToHost, stream_),
             "loss");
  cuda_check(cudaStreamSynchronize(stream_), "indicator training");
  return loss / static_cast<double>(batch);
}

double MlpTrainer::gradient(const float *features, const std::uint8_t *labels, std::int64_t n,
                            double pos_weight, float *grad_out) {
  if (n <= 0 || n % kMlpBatch != 0)
    throw SolverError(WASL_ERR_ARGUMENT, "indicator gradient: samples must be a positive"
                                         " multiple of 64");
  DeviceArray<float> f(static_cast<std::size_t>(n) * shape_.features), g(shape_.count);
  DeviceArray<std::uint8_t> y(n);
  cuda_check(cudaMemcpyAsync(f.get(), features, sizeof(float) * n * shape_.features,
                             cudaMemcpyHostToDevice, stream_),
             "gradient data");
  cuda_check(cudaMemcpyAsync(y.get(), labels, n, cudaMemcpyHostToDevice, stream_), "labels");
  cuda_check(cudaMemsetAsync(g.get(), 0, sizeof(float) * shape_.count, stream_), "grad reset");
  cuda_check(cudaMemsetAsync(loss_.get(), 0, sizeof(double), stream_), "loss reset");
  launch_mlp_train(shape_, params_.get(), f.get(), y.get(), n, 0, n / kMlpBatch,
                   static_cast<float>(pos_weight), g.get(), loss_.get(), stream_);
  double loss = 0.0;
  cuda_check(cudaMemcpyAsync(grad_out, g.get(), sizeof(float) * shape_.count,
                             cudaMemcpyDeviceToHost, stream_),
             "gradient");
  cuda_check(cudaMemcpyAsync(&loss, loss_.get(), sizeof(double), cudaMemcpyDeviceToHost, stream_),
             "loss");
  cuda_check(cudaStreamSynchronize(stream_), "indicator gradient");
  for (std::int64_t i = 0; i < shape_.count; ++i)
    grad_out[i] /= static_cast<float>(n);
  return loss / static_cast<double>(n);
}

void MlpTrainer::predict(const float *features, std::int64_t n, float *logits) {
  DeviceArray<float> f(static_cast<std::size_t>(n) * shape_.features), z(n);
  cuda_check(cudaMemcpyAsync(f.get(), features, sizeof(float) * n * shape_.features,
                             cudaMemcpyHostToDevice, stream_),
             "predict data");
  launch_mlp_predict(shape_, params_.get(), f.get(), n, z.get(), stream_);
  cuda_check(cudaMemcpyAsync(logits, z.get(), sizeof(float) * n, cudaMemcpyDeviceToHost, stream_),
             "logits");
  cuda_check(cudaStreamSynchronize(stream_), "indicator predict");
}

void MlpTrainer::get(float *params) const {
  cuda_check(cudaMemcpyAsync(params, params_.get(), sizeof(float) * shape_.count,
                             cudaMemcpyDeviceToHost, stream_),
             "weights");
  cuda_check(cudaStreamSynchronize(stream_), "weights");
}

void MlpTrainer::set(const float *params) {
  cuda_check(cudaMemcpyAsync(params_.get(), params, sizeof(float) * shape_.count,
                             cudaMemcpyHostToDevice, stream_),
             "weights");
  cuda_check(cudaStreamSynchronize(stream_), "weights");
}

} // namespace wasl_b200

struct wasl_mlp {
  std::unique_ptr<wasl_b200::MlpTrainer> trainer;
  std::string error;
};

namespace {

template <typename F> int guarded(wasl_mlp *h, F &&body) {
  if (!h)
    return WASL_ERR_ARGUMENT;
  try {
    body();
    h->error.clear();
    return WASL_OK;
  } catch (const wasl_b200::SolverError &e) {
    h->error = e.what();
    return e.status;
  } catch (const std::invalid_argument &e) {
    h->error = e.what();
    return WASL_ERR_ARGUMENT;
  } catch (const std::exception &e) {
    h->error = e.what();
    return WASL_ERR_RUNTIME;
  }
}

} // namespace

extern "C" {

int wasl_mlp_create(int features, uint64_t seed, int device, wasl_mlp **handle, char *error,
                    size_t error_length) {
  if (!handle)
    return WASL_ERR_ARGUMENT;
  *handle = nullptr;
  try {
    auto *h = new wasl_mlp;
    try {
      h->trainer = std::make_unique<wasl_b200::MlpTrainer>(features, seed, device);
    } catch (...) {
      delete h;
      throw;
    }
    *handle = h;
    return WASL_OK;
  } catch (const std::exception &e) {
    if (error && error_length) {
      std::strncpy(error, e.what(), error_length - 1);
      error[error_length - 1] = '\0';
    }
    const auto *se = dynamic_cast<const wasl_b200::SolverError *>(&e);
    return se ? se->status
              : (dynamic_cast<const std::invalid_argument *>(&e) ? WASL_ERR_ARGUMENT
                                                                 : WASL_ERR_RUNTIME);
  }
}

void wasl_mlp_destroy(wasl_mlp *h) { delete h; }

const char *wasl_mlp_last_error(const wasl_mlp *h) { return h ? h->error.c_str() : "null handle"; }

int wasl_mlp_parameter_count(const wasl_mlp *h, int64_t *count) {
  return guarded(const_cast<wasl_mlp *>(h), [&] { *count = h->trainer->shape().count; });
}

int wasl_mlp_set_data(wasl_mlp *h, const float *features, const uint8_t *labels, int64_t count) {
  return guarded(h, [&] {
    if (!features || !labels)
      throw wasl_b200::SolverError(WASL_ERR_ARGUMENT, "indicator data: null argument");
    h->trainer->set_data(features, labels, count);
  });
}

int wasl_mlp_train(wasl_mlp *h, int64_t steps, int64_t batch, double learning_rate,
                   double positive_weight, double *loss) {
  return guarded(h, [&] {
    const double l = h->trainer->train(steps, batch, learning_rate, positive_weight);
    if (loss)
      *loss = l;
  });
}

int wasl_mlp_gradient(wasl_mlp *h, const float *features, const uint8_t *labels, int64_t count,
                      double positive_weight, float *gradient, double *loss) {
  return guarded(h, [&] {
    const double l = h->trainer->gradient(features, labels, count, positive_weight, gradient);
    if (loss)
      *loss = l;
  });
}

int wasl_mlp_predict(wasl_mlp *h, const float *features, int64_t count, float *logits) {
  return guarded(h, [&] { h->trainer->predict(features, count, logits); });
}

int wasl_mlp_get_weights(const wasl_mlp *h, float *weights, int64_t count) {
  return guarded(const_cast<wasl_mlp *>(h), [&] {
    if (count != h->trainer->shape().count)
      throw wasl_b200::SolverError(WASL_ERR_ARGUMENT, "indicator weights: wrong count");
    h->trainer->get(weights);
  });
}

int wasl_mlp_set_weights(wasl_mlp *h, const float *weights, int64_t count) {
  return guarded(h, [&] {
    if (count != h->trainer->shape().count)
      throw wasl_b200::SolverError(WASL_ERR_ARGUMENT, "indicator weights: wrong count");
    h->trainer->set(weights);
  });
}

} // extern "C"
