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
  const double *uploaded_ = nullptr; // the host vector stable_time_step just uploaded
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

} // namespace wasl_b200

// C twins of the reference bridge's coarse functions
// (crates/wasl-bridge/include/bridge.hpp:7-32, defined at
// crates/wasl-bridge/src/bridge.cpp:79-216), so the Rust `ffi` block can bind
// them directly: rust::Str becomes a NUL-terminated const char *,
// rust::Slice<const T> a pointer and its length (element count, as
// Slice::size()), rust::Slice<const rust::String> an array of const char *,
// `bool` an int, and the returned rust::String is written to `summary`
// (truncated to summary_length - 1 bytes, NUL-terminated).  Every twin returns
// 0 on success; on failure -2 with the reference's message (the
// std::exception text cxx would turn into Err) in `error`.  They run the
// reference's own case code; the solver runs use the GPU-backed models above.
extern "C" {
// run_euler_case (bridge.hpp:24-32) on the plain FP64 GPU path: the drop-in.
// regions: 10 doubles per region (shape 0 default, 1 interval, 2 circle;
// lower, upper, centre x, centre y, radius; density, velocity x, velocity y,
// pressure); boundary kinds 0 periodic, 1 inflow, 2 outflow.
int wasl_run_euler_case_gpu(const char *mesh_path, const char *output_path,
                            const char *restart_path, int limiting, double sensor_threshold,
                            double density_floor, double pressure_floor, int dimensions,
                            int polynomial_order, double heat_capacity_ratio, double cfl,
                            double start_time, double end_time, std::uint64_t max_steps,
                            std::uint64_t history_interval, std::uint64_t visualization_interval,
                            std::uint64_t checkpoint_interval, std::uint64_t keep_checkpoints,
                            const double *regions, std::size_t regions_length,
                            const char *const *boundary_names, const std::uint8_t *boundary_kinds,
                            const double *boundary_values, std::size_t boundary_count,
                            char *summary, std::size_t summary_length, char *error,
                            std::size_t error_length);

// wasl_run_euler_case_gpu with a choice of precision form (enum
// wasl_precision; WASL_PLAIN_FP64 gives wasl_run_euler_case_gpu).  No
// counterpart in the bridge.
int wasl_run_euler_case_gpu_ex(
    const char *mesh_path, const char *output_path, const char *restart_path, int limiting,
    double sensor_threshold, double density_floor, double pressure_floor, int dimensions,
    int polynomial_order, double heat_capacity_ratio, double cfl, double start_time,
    double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, const double *regions, std::size_t regions_length,
    const char *const *boundary_names, const std::uint8_t *boundary_kinds,
    const double *boundary_values, std::size_t boundary_count, int precision, char *summary,
    std::size_t summary_length, char *error, std::size_t error_length);

// run_scalar_advection_case (bridge.hpp:13-22) on the GPU: intervals 3
// doubles each (lower, upper, value), circles 4 (centre x, centre y, radius,
// value).  mpi on a line mesh fails as the reference's non-MPI build does
// ("simulation: bridge was built without MPI support"); on triangles it is
// ignored, as the reference ignores it.
int wasl_run_scalar_advection_case_gpu(
    const char *mesh_path, const char *output_path, const char *restart_path, int mpi,
    int dimensions, int polynomial_order, double velocity_x, double velocity_y, double cfl,
    double start_time, double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, double initial_default, int initial_sine,
    double initial_sine_amplitude, const double *intervals, std::size_t intervals_length,
    const double *circles, std::size_t circles_length, const char *const *boundary_names,
    const std::uint8_t *boundary_kinds, const double *boundary_values,
    std::size_t boundary_count, char *summary, std::size_t summary_length, char *error,
    std::size_t error_length);

// inspect_checkpoint, inspect_prepared_mesh, export_checkpoint, prepare_mesh
// and prepare_mpi_run_directory (bridge.hpp:7-11): host file utilities, the
// reference's own code behind the same C conventions.
int wasl_inspect_checkpoint(const char *checkpoint_path, char *summary,
                            std::size_t summary_length, char *error, std::size_t error_length);
int wasl_inspect_prepared_mesh(const char *mesh_path, char *summary, std::size_t summary_length,
                               char *error, std::size_t error_length);
int wasl_export_checkpoint(const char *checkpoint_path, const char *mesh_path,
                           const char *output_path, char *summary, std::size_t summary_length,
                           char *error, std::size_t error_length);
int wasl_prepare_mesh(const char *source_path, const char *output_path, char *summary,
                      std::size_t summary_length, char *error, std::size_t error_length);
int wasl_prepare_mpi_run_directory(const char *root_path, const char *effective_config,
                                   char *summary, std::size_t summary_length, char *error,
                                   std::size_t error_length);
}
