// Kernel accounting of a solver handle (launch counts and stage-kernel timing).
#include "solver.hpp"

namespace wasl_b200 {

void Solver::profile_begin() {
  profiling_ = true;
  launches_ = 0;
  events_used_ = 0;
}

void Solver::stage_begin() {
  if (!profiling_)
    return;
  if (events_used_ + 2 > events_.size())
    for (int k = 0; k < 64; ++k) {
      cudaEvent_t ev;
      cuda_check(cudaEventCreate(&ev), "event");
      events_.push_back(ev);
    }
  cuda_check(cudaEventRecord(events_[events_used_++], stream_), "event record");
}

void Solver::stage_end() {
  if (!profiling_)
    return;
  cuda_check(cudaEventRecord(events_[events_used_++], stream_), "event record");
}

void Solver::profile_end(double &stage_ms, std::int64_t &stage_kernels, std::int64_t &launches) {
  cuda_check(cudaStreamSynchronize(stream_), "profile");
  stage_ms = 0.0;
  stage_split_[0] = stage_split_[1] = stage_split_[2] = 0.0;
  for (std::size_t k = 0; k + 1 < events_used_; k += 2) {
    float ms = 0.0f;
    cuda_check(cudaEventElapsedTime(&ms, events_[k], events_[k + 1]), "elapsed");
    stage_ms += ms;
    stage_split_[(k / 2) % 3] += ms; // stage kernels come in SSP-RK3 triples
  }
  stage_kernels = static_cast<std::int64_t>(events_used_ / 2);
  launches = launches_;
  profiling_ = false;
  events_used_ = 0;
}

Solver::~Solver() {
  for (cudaEvent_t ev : events_)
    cudaEventDestroy(ev);
}

} // namespace wasl_b200
