// GpuEulerModel and run_euler_case_gpu (see serial_case_model.hpp).
#include "serial_case_model.hpp"

#include <algorithm>
#include <cstring>
#include <exception>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "case/euler_drivers.hpp"
#include "case/line_boundary_resolution.hpp"
#include "case/scalar_advection_drivers.hpp"
#include "wasl/basis/mode_count.hpp"
#include "wasl/case/case_validation.hpp"
#include "wasl/case/initial_state.hpp"
#include "wasl/equations/euler/euler.hpp"
#include "wasl/mesh/prepared/mesh_from_prepared.hpp"

namespace wasl_b200 {

GpuEulerModel::GpuEulerModel(const wasl::EulerCase &config, const wasl::CaseMesh &mesh,
                             int precision)
    : config_(config) {
  // The handle takes the mesh as node tags, coordinates and element nodes, in
  // the mesh's own element and node order (it normalizes them as the
  // reference does, so faces come out in the reference's order).
  wasl_gpu_config cfg;
  wasl_gpu_config_default(&cfg);
  cfg.dimensions = config.dimensions;
  std::map<std::int64_t, std::pair<double, double>> nodes;
  std::vector<std::int64_t> element_nodes;
  std::size_t elements = 0;
  if (config.dimensions == 1) {
    line_ = wasl::line_mesh_from_prepared(mesh.prepared);
    elements = line_.elements.size();
    for (const auto &el : line_.elements) {
      nodes.emplace(el.left_node, std::make_pair(el.x_left, 0.0));
      nodes.emplace(el.right_node, std::make_pair(el.x_right, 0.0));
      element_nodes.push_back(el.left_node);
      element_nodes.push_back(el.right_node);
    }
    // Periodic or outflow ends, resolved from the named boundaries as the
    // reference resolves them (inflow is rejected for Euler).
    const auto ends = wasl::resolve_line_boundaries(mesh.prepared, line_, config.boundaries);
    const auto kind = [](const wasl::BoundaryCondition &b) {
      if (b.kind == wasl::BoundaryKind::inflow)
        throw std::runtime_error("simulation: Euler inflow boundaries are not supported");
      return b.kind == wasl::BoundaryKind::periodic ? WASL_PERIODIC : WASL_OUTFLOW;
    };
    cfg.boundary_left = kind(ends.left);
    cfg.boundary_right = kind(ends.right);
  } else {
    triangles_ = wasl::triangle_mesh_from_prepared(mesh.prepared);
    elements = triangles_.elements.size();
    for (const auto &el : triangles_.elements) {
      const std::int64_t tags[3] = {el.node0, el.node1, el.node2};
      const double xy[3][2] = {{el.x0, el.y0}, {el.x1, el.y1}, {el.x2, el.y2}};
      for (int k = 0; k < 3; ++k) {
        nodes.emplace(tags[k], std::make_pair(xy[k][0], xy[k][1]));
        element_nodes.push_back(tags[k]);
      }
    }
  }
  std::vector<std::int64_t> node_tags;
  std::vector<double> coordinates;
  for (const auto &[tag, xy] : nodes) {
    node_tags.push_back(tag);
    coordinates.push_back(xy.first);
    if (config.dimensions == 2)
      coordinates.push_back(xy.second);
  }

  cfg.equation = WASL_EULER;
  cfg.polynomial_order = config.polynomial_order;
  cfg.heat_capacity_ratio = config.heat_capacity_ratio;
  cfg.limiting = config.limiting ? 1 : 0;
  cfg.sensor_threshold = config.sensor_threshold;
  cfg.density_floor = config.density_floor;
  cfg.pressure_floor = config.pressure_floor;
  cfg.precision = precision;
  char error[512] = {0};
  if (wasl_gpu_create(&cfg, static_cast<std::int64_t>(node_tags.size()), node_tags.data(),
                      coordinates.data(), static_cast<std::int64_t>(elements),
                      element_nodes.data(), &gpu_, error, sizeof error) != 0)
    throw std::runtime_error(error);

  const wasl::Euler equation{config.heat_capacity_ratio};
  const double cfl = config.cfl;
  model_.variable_count = wasl::Euler::variable_count;
  model_.mode_count = config.dimensions == 1 ? wasl::line_mode_count(config.polynomial_order)
                                             : wasl::triangle_mode_count(config.polynomial_order);
  // Layouts, mass and cell averages are host work on the state of record:
  // the reference's own operations.
  if (config.dimensions == 1)
    wasl::add_euler_state_operations(model_, line_);
  else
    wasl::add_euler_state_operations(model_, triangles_);
  const auto size = [](const wasl::SerialCaseModel::State &s) {
    return static_cast<std::int64_t>(s.size());
  };
  model_.initial_state = [this, equation, size] {
    auto state = config_.dimensions == 1
                     ? wasl::initial_coefficients(line_, config_, equation)
                     : wasl::initial_coefficients(triangles_, config_, equation);
    check(wasl_gpu_set_state(gpu_, state.data(), size(state)));
    check(wasl_gpu_limit(gpu_)); // the reference limits the projected state
    check(wasl_gpu_get_state(gpu_, state.data(), size(state)));
    return state;
  };
  model_.stable_time_step = [this, cfl, size](const wasl::SerialCaseModel::State &state) {
    double dt = 0.0;
    check(wasl_gpu_set_state(gpu_, state.data(), size(state)));
    check(wasl_gpu_stable_dt(gpu_, cfl, &dt));
    return dt;
  };
  model_.advance = [this, size](double dt, wasl::SerialCaseModel::State &state,
                                wasl::SspRk3Workspace &) {
    check(wasl_gpu_set_state(gpu_, state.data(), size(state)));
    check(wasl_gpu_step(gpu_, dt));
    check(wasl_gpu_get_state(gpu_, state.data(), size(state)));
  };
}

GpuEulerModel::~GpuEulerModel() { wasl_gpu_destroy(gpu_); }

void GpuEulerModel::check(int status) const {
  if (status != 0)
    throw std::runtime_error(wasl_gpu_last_error(gpu_));
}

wasl::SimulationSummary run_euler_case_gpu(const wasl::EulerCase &config, int precision) {
  wasl::validate_euler_case(config);
  if (config.dimensions == 2 && !wasl::all_periodic(config.boundaries))
    throw std::runtime_error("simulation: 2D Euler boundaries must be periodic");
  const auto mesh = wasl::load_case_mesh(config.files.prepared_mesh, config.dimensions);
  const GpuEulerModel gpu(config, mesh, precision);
  return wasl::run_serial_case(config.files, config.run, mesh, gpu.model());
}

GpuScalarAdvectionModel::GpuScalarAdvectionModel(const wasl::ScalarAdvectionCase &config,
                                                 const wasl::CaseMesh &mesh)
    : config_(config) {
  wasl_gpu_config cfg;
  wasl_gpu_config_default(&cfg);
  cfg.dimensions = config.dimensions;
  cfg.equation = WASL_SCALAR_ADVECTION;
  cfg.polynomial_order = config.polynomial_order;
  cfg.velocity_x = config.wavespeed;
  cfg.velocity_y = config.velocity_y;
  std::map<std::int64_t, std::pair<double, double>> nodes;
  std::vector<std::int64_t> element_nodes;
  std::size_t elements = 0;
  if (config.dimensions == 1) {
    line_ = wasl::line_mesh_from_prepared(mesh.prepared);
    elements = line_.elements.size();
    for (const auto &el : line_.elements) {
      nodes.emplace(el.left_node, std::make_pair(el.x_left, 0.0));
      nodes.emplace(el.right_node, std::make_pair(el.x_right, 0.0));
      element_nodes.push_back(el.left_node);
      element_nodes.push_back(el.right_node);
    }
    const auto ends = wasl::resolve_line_boundaries(mesh.prepared, line_, config.boundaries);
    const auto kind = [](const wasl::BoundaryCondition &b) {
      return b.kind == wasl::BoundaryKind::periodic  ? WASL_PERIODIC
             : b.kind == wasl::BoundaryKind::inflow ? WASL_INFLOW
                                                    : WASL_OUTFLOW;
    };
    cfg.boundary_left = kind(ends.left);
    cfg.boundary_right = kind(ends.right);
    cfg.inflow_left = ends.left.value;
    cfg.inflow_right = ends.right.value;
  } else {
    triangles_ = wasl::triangle_mesh_from_prepared(mesh.prepared);
    elements = triangles_.elements.size();
    for (const auto &el : triangles_.elements) {
      const std::int64_t tags[3] = {el.node0, el.node1, el.node2};
      const double xy[3][2] = {{el.x0, el.y0}, {el.x1, el.y1}, {el.x2, el.y2}};
      for (int k = 0; k < 3; ++k) {
        nodes.emplace(tags[k], std::make_pair(xy[k][0], xy[k][1]));
        element_nodes.push_back(tags[k]);
      }
    }
  }
  std::vector<std::int64_t> node_tags;
  std::vector<double> coordinates;
  for (const auto &[tag, xy] : nodes) {
    node_tags.push_back(tag);
    coordinates.push_back(xy.first);
    if (config.dimensions == 2)
      coordinates.push_back(xy.second);
  }
  char error[512] = {0};
  if (wasl_gpu_create(&cfg, static_cast<std::int64_t>(node_tags.size()), node_tags.data(),
                      coordinates.data(), static_cast<std::int64_t>(elements),
                      element_nodes.data(), &gpu_, error, sizeof error) != 0)
    throw std::runtime_error(error);
  check(wasl_gpu_stable_dt(gpu_, config.cfl, &step_)); // independent of the state

  model_.variable_count = 1;
  model_.mode_count = config.dimensions == 1 ? wasl::line_mode_count(config.polynomial_order)
                                             : wasl::triangle_mode_count(config.polynomial_order);
  if (config.dimensions == 1)
    wasl::add_scalar_state_operations(model_, line_);
  else
    wasl::add_scalar_state_operations(model_, triangles_);
  model_.initial_state = [this] {
    return config_.dimensions == 1 ? wasl::initial_coefficients(line_, config_)
                                   : wasl::initial_coefficients(triangles_, config_);
  };
  model_.stable_time_step = [this](const wasl::SerialCaseModel::State &) { return step_; };
  model_.advance = [this](double dt, wasl::SerialCaseModel::State &state,
                          wasl::SspRk3Workspace &) {
    // The handle holds U[mode][element], the reference's checkpoint layout.
    auto persisted = model_.to_checkpoint(state);
    const auto n = static_cast<std::int64_t>(persisted.size());
    check(wasl_gpu_set_state(gpu_, persisted.data(), n));
    check(wasl_gpu_step(gpu_, dt));
    check(wasl_gpu_get_state(gpu_, persisted.data(), n));
    state = model_.from_checkpoint(persisted);
  };
}

GpuScalarAdvectionModel::~GpuScalarAdvectionModel() { wasl_gpu_destroy(gpu_); }

void GpuScalarAdvectionModel::check(int status) const {
  if (status != 0)
    throw std::runtime_error(wasl_gpu_last_error(gpu_));
}

wasl::SimulationSummary run_scalar_advection_case_gpu(const wasl::ScalarAdvectionCase &config) {
  wasl::validate_scalar_advection_case(config);
  if (config.mpi)
    throw std::runtime_error("run_scalar_advection_case_gpu: MPI runs are not on the GPU path");
  if (config.dimensions == 2 && !wasl::all_periodic(config.boundaries))
    throw std::runtime_error("simulation: 2D scalar-advection boundaries must be periodic");
  const auto mesh = wasl::load_case_mesh(config.files.prepared_mesh, config.dimensions);
  const GpuScalarAdvectionModel gpu(config, mesh);
  return wasl::run_serial_case(config.files, config.run, mesh, gpu.model());
}

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
                                          std::size_t region_count) {
  wasl::EulerCase c;
  c.files = {prepared_mesh, output_directory, restart ? restart : ""};
  c.run = {start_time,           end_time,           max_steps,       history_interval,
           visualization_interval, checkpoint_interval, keep_checkpoints};
  c.limiting = limiting != 0;
  c.sensor_threshold = sensor_threshold;
  c.density_floor = density_floor;
  c.pressure_floor = pressure_floor;
  c.dimensions = dimensions;
  c.polynomial_order = polynomial_order;
  c.heat_capacity_ratio = heat_capacity_ratio;
  c.cfl = cfl;
  for (std::size_t i = 0; i < region_count; ++i) {
    const double *r = regions + 10 * i;
    wasl::EulerRegion region;
    const int shape = static_cast<int>(r[0]);
    region.shape = shape == 1   ? wasl::EulerRegion::Shape::interval
                   : shape == 2 ? wasl::EulerRegion::Shape::circle
                                : wasl::EulerRegion::Shape::default_region;
    region.lower = r[1];
    region.upper = r[2];
    region.center_x = r[3];
    region.center_y = r[4];
    region.radius = r[5];
    region.value = {r[6], r[7], r[8], r[9]};
    c.initial_regions.push_back(region);
  }
  return c;
}

} // namespace wasl_b200

extern "C" int wasl_run_euler_case_gpu(
    const char *prepared_mesh, const char *output_directory, const char *restart, int limiting,
    double sensor_threshold, double density_floor, double pressure_floor, int dimensions,
    int polynomial_order, double heat_capacity_ratio, double cfl, double start_time,
    double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, const double *regions, std::size_t region_count,
    int precision, std::uint64_t *steps, double *time, char *error, std::size_t error_length) {
  try {
    const auto config = wasl_b200::euler_case_from_arguments(
        prepared_mesh, output_directory, restart, limiting, sensor_threshold, density_floor,
        pressure_floor, dimensions, polynomial_order, heat_capacity_ratio, cfl, start_time,
        end_time, max_steps, history_interval, visualization_interval, checkpoint_interval,
        keep_checkpoints, regions, region_count);
    const auto summary = wasl_b200::run_euler_case_gpu(config, precision);
    if (steps)
      *steps = summary.step;
    if (time)
      *time = summary.time;
    return 0;
  } catch (const std::exception &e) {
    if (error && error_length) {
      std::strncpy(error, e.what(), error_length - 1);
      error[error_length - 1] = '\0';
    }
    return -2;
  }
}

extern "C" int wasl_run_scalar_advection_case_gpu(
    const char *prepared_mesh, const char *output_directory, const char *restart,
    int dimensions, int polynomial_order, double velocity_x, double velocity_y, double cfl,
    double start_time, double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, double initial_default, int initial_sine,
    double initial_sine_amplitude, const double *intervals, std::size_t interval_count,
    const double *circles, std::size_t circle_count, std::uint64_t *steps, double *time,
    char *error, std::size_t error_length) {
  try {
    wasl::ScalarAdvectionCase c;
    c.files = {prepared_mesh, output_directory, restart ? restart : ""};
    c.run = {start_time,           end_time,           max_steps,       history_interval,
             visualization_interval, checkpoint_interval, keep_checkpoints};
    c.dimensions = dimensions;
    c.polynomial_order = polynomial_order;
    c.wavespeed = velocity_x;
    c.velocity_y = velocity_y;
    c.cfl = cfl;
    c.initial_default = initial_default;
    c.initial_sine = initial_sine != 0;
    c.initial_sine_amplitude = initial_sine_amplitude;
    for (std::size_t i = 0; i < interval_count; ++i)
      c.initial_intervals.push_back({intervals[3 * i], intervals[3 * i + 1], intervals[3 * i + 2]});
    for (std::size_t i = 0; i < circle_count; ++i)
      c.initial_circles.push_back(
          {circles[4 * i], circles[4 * i + 1], circles[4 * i + 2], circles[4 * i + 3]});
    const auto summary = wasl_b200::run_scalar_advection_case_gpu(c);
    if (steps)
      *steps = summary.step;
    if (time)
      *time = summary.time;
    return 0;
  } catch (const std::exception &e) {
    if (error && error_length) {
      std::strncpy(error, e.what(), error_length - 1);
      error[error_length - 1] = '\0';
    }
    return -2;
  }
}
