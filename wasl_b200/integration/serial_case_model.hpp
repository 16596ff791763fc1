// A SerialCaseModel backed by the GPU handle, for the reference's own run loop.
//
// The reference runs every case through run_serial_case
// (cpp/src/case/serial_case_runner.cpp:107-149), which owns time, restart,
// history, snapshots and checkpoint rotation, and calls a SerialCaseModel
// (cpp/include/wasl/case/serial_case_runner.hpp:22-34) for the numerics.
// GpuEulerModel is that model with its numerics on the GPU through the C-ABI
// (include/wasl_b200.h), on a line or triangle mesh: the host vector stays the
// state of record, and each stable_time_step / advance copies it in and out.
// run_euler_case_gpu is run_euler_case (cpp/src/case/euler_case.cpp:7-11, with
// cpp/src/case/euler_line.cpp:14-47 and cpp/src/case/euler_triangle.cpp:15-50)
// with this model: same validation, boundaries, files and outputs.  This file builds against the reference's headers and
// library; it is the piece a maintainer adds to the reference's tree.
#pragma once

#include <cstddef>
#include <cstdint>

#include "wasl/case/case_mesh.hpp"
#include "wasl/case/euler_case.hpp"
#include "wasl/case/scalar_advection_case.hpp"
#include "wasl/case/serial_case_runner.hpp"
#include "wasl/case/simulation_summary.hpp"
#include "wasl/mesh/line/line_mesh.hpp"
#include "wasl/mesh/triangle/triangle_mesh.hpp"
#include "wasl_b200.h"

namespace wasl_b200 {

class GpuEulerModel {
public:
  // precision: enum wasl_precision (WASL_PLAIN_FP64 is the bit-consistent drop-in).
  GpuEulerModel(const wasl::EulerCase &config, const wasl::CaseMesh &mesh, int precision);
  ~GpuEulerModel();
  GpuEulerModel(const GpuEulerModel &) = delete;
  GpuEulerModel &operator=(const GpuEulerModel &) = delete;

  const wasl::SerialCaseModel &model() const { return model_; }

private:
  void check(int status) const;

  wasl_gpu *gpu_ = nullptr;
  wasl::EulerCase config_;
  wasl::LineMesh line_;          // dimensions 1
  wasl::TriangleMesh triangles_; // dimensions 2
  wasl::SerialCaseModel model_;
};

wasl::SimulationSummary run_euler_case_gpu(const wasl::EulerCase &config, int precision);

// Scalar advection: the same on the plain FP64 GPU path.  The reference's
// state of record is element-major (U[element][mode]); the model converts it
// with the reference's own checkpoint layout operations around each GPU call.
// The time step is fixed at setup, as the reference fixes it
// (cpp/src/case/scalar_advection_line.cpp:14-17,
// cpp/src/case/scalar_advection_triangle.cpp:21-22).
class GpuScalarAdvectionModel {
public:
  GpuScalarAdvectionModel(const wasl::ScalarAdvectionCase &config, const wasl::CaseMesh &mesh);
  ~GpuScalarAdvectionModel();
  GpuScalarAdvectionModel(const GpuScalarAdvectionModel &) = delete;
  GpuScalarAdvectionModel &operator=(const GpuScalarAdvectionModel &) = delete;

  const wasl::SerialCaseModel &model() const { return model_; }

private:
  void check(int status) const;

  wasl_gpu *gpu_ = nullptr;
  wasl::ScalarAdvectionCase config_;
  wasl::LineMesh line_;
  wasl::TriangleMesh triangles_;
  wasl::SerialCaseModel model_;
  double step_ = 0.0;
};

// run_scalar_advection_case (cpp/src/case/scalar_advection_case.cpp) with the
// GPU model, for serial runs (the two-rank MPI driver is not on this path).
wasl::SimulationSummary run_scalar_advection_case_gpu(const wasl::ScalarAdvectionCase &config);

// The bridge's flat run_euler_case arguments (crates/wasl-bridge/include/bridge.hpp:24-32)
// for a periodic case (empty boundary list): each region is 10 doubles (shape 0 default, 1 interval,
// 2 circle; lower, upper, centre x, centre y, radius; density, velocity x,
// velocity y, pressure).
wasl::EulerCase euler_case_from_arguments(const char *prepared_mesh, const char *output_directory,
                                          const char *restart, int limiting,
                                          double sensor_threshold, double density_floor,
                                          double pressure_floor, int dimensions,
                                          int polynomial_order, double heat_capacity_ratio,
                                          double cfl, double start_time, double end_time,
                                          std::uint64_t max_steps, std::uint64_t history_interval,
                                          std::uint64_t visualization_interval,
                                          std::uint64_t checkpoint_interval,
                                          std::uint64_t keep_checkpoints, const double *regions,
                                          std::size_t region_count);

} // namespace wasl_b200

extern "C" {
// run_euler_case_gpu from flat arguments (as euler_case_from_arguments); 0 on
// success with the summary's step count and final time, else -2 with the
// reference's message in `error`.
int wasl_run_euler_case_gpu(const char *prepared_mesh, const char *output_directory,
                            const char *restart, int limiting, double sensor_threshold,
                            double density_floor, double pressure_floor, int dimensions,
                            int polynomial_order, double heat_capacity_ratio, double cfl,
                            double start_time, double end_time, std::uint64_t max_steps,
                            std::uint64_t history_interval, std::uint64_t visualization_interval,
                            std::uint64_t checkpoint_interval, std::uint64_t keep_checkpoints,
                            const double *regions, std::size_t region_count, int precision,
                            std::uint64_t *steps, double *time, char *error,
                            std::size_t error_length);

// run_scalar_advection_case_gpu from the bridge's flat arguments
// (crates/wasl-bridge/include/bridge.hpp:13-22) for a periodic serial case:
// intervals are 3 doubles each (lower, upper, value), circles 4 (centre x,
// centre y, radius, value).  Statuses as wasl_run_euler_case_gpu.
int wasl_run_scalar_advection_case_gpu(
    const char *prepared_mesh, const char *output_directory, const char *restart,
    int dimensions, int polynomial_order, double velocity_x, double velocity_y, double cfl,
    double start_time, double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, double initial_default, int initial_sine,
    double initial_sine_amplitude, const double *intervals, std::size_t interval_count,
    const double *circles, std::size_t circle_count, std::uint64_t *steps, double *time,
    char *error, std::size_t error_length);
}
