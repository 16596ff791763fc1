// GpuEulerModel and run_euler_case_gpu (see serial_case_model.hpp).
#include "serial_case_model.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <map>
#include <sstream>
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
#include "wasl/case/mpi_run_directory.hpp"
#include "wasl/io/checkpoint_file.hpp"
#include "wasl/io/prepared_mesh_file.hpp"
#include "wasl/io/vtu_writer.hpp"
#include "wasl/mesh/line/build_line_mesh.hpp"
#include "wasl/mesh/msh/msh_reader.hpp"
#include "wasl/mesh/prepared/mesh_from_prepared.hpp"
#include "wasl/mesh/prepared/prepare_mesh.hpp"
#include "wasl/mesh/triangle/build_triangle_mesh.hpp"

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
  // run_serial_case calls advance right after stable_time_step on the same
  // state (cpp/src/case/serial_case_runner.cpp:127-129), so the state that
  // stable_time_step uploaded is still on the device: advance uploads only a
  // vector other than that one.
  model_.stable_time_step = [this, cfl, size](const wasl::SerialCaseModel::State &state) {
    double dt = 0.0;
    check(wasl_gpu_set_state(gpu_, state.data(), size(state)));
    uploaded_ = state.data();
    check(wasl_gpu_stable_dt(gpu_, cfl, &dt));
    return dt;
  };
  model_.advance = [this, size](double dt, wasl::SerialCaseModel::State &state,
                                wasl::SspRk3Workspace &) {
    if (state.data() != uploaded_)
      check(wasl_gpu_set_state(gpu_, state.data(), size(state)));
    uploaded_ = nullptr;
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
  if (config.dimensions == 2 && !wasl::all_periodic(config.boundaries))
    throw std::runtime_error("simulation: 2D scalar-advection boundaries must be periodic");
  const auto mesh = wasl::load_case_mesh(config.files.prepared_mesh, config.dimensions);
  // The reference's distributed line driver, in a build without MPI
  // (cpp/src/case/scalar_advection_distributed.cpp:286-289); triangles ignore
  // the flag (cpp/src/case/scalar_advection_case.cpp:10-15).
  if (config.dimensions == 1 && config.mpi)
    throw std::runtime_error("simulation: bridge was built without MPI support");
  const GpuScalarAdvectionModel gpu(config, mesh);
  return wasl::run_serial_case(config.files, config.run, mesh, gpu.model());
}

namespace {

void write_text(const std::string &text, char *out, std::size_t length) {
  if (out && length) {
    std::strncpy(out, text.c_str(), length - 1);
    out[length - 1] = '\0';
  }
}

// The bridge's summary string (crates/wasl-bridge/src/bridge.cpp:39-45).
std::string summary_message(const wasl::SimulationSummary &summary) {
  std::ostringstream message;
  message.precision(17);
  message << "step=" << summary.step << " time=" << summary.time
          << " checkpoint=" << summary.checkpoint.string();
  return message.str();
}

// The bridge's named boundaries (bridge.cpp:48-62); one length for the three
// parallel arrays, so only the kind needs checking.
std::vector<wasl::NamedBoundary> named_boundaries(const char *const *names,
                                                  const std::uint8_t *kinds,
                                                  const double *values, std::size_t count) {
  std::vector<wasl::NamedBoundary> boundaries;
  if (count && (!names || !kinds || !values))
    throw std::runtime_error("boundaries: invalid boundary data");
  for (std::size_t i = 0; i < count; ++i) {
    if (!names[i] || kinds[i] > static_cast<std::uint8_t>(wasl::BoundaryKind::outflow))
      throw std::runtime_error("boundaries: invalid boundary kind");
    boundaries.push_back({names[i], {static_cast<wasl::BoundaryKind>(kinds[i]), values[i]}});
  }
  return boundaries;
}

wasl::CaseFiles case_files(const char *mesh, const char *output, const char *restart) {
  if (!mesh || !output)
    throw std::runtime_error("files: mesh and output paths are required");
  return {mesh, output, restart ? restart : ""};
}

template <typename Body>
int twin(char *summary, std::size_t summary_length, char *error, std::size_t error_length,
         Body &&body) {
  try {
    write_text(body(), summary, summary_length);
    return 0;
  } catch (const std::exception &e) {
    write_text(e.what(), error, error_length);
    return -2;
  }
}

} // namespace
} // namespace wasl_b200

extern "C" int wasl_run_euler_case_gpu_ex(
    const char *mesh_path, const char *output_path, const char *restart_path, int limiting,
    double sensor_threshold, double density_floor, double pressure_floor, int dimensions,
    int polynomial_order, double heat_capacity_ratio, double cfl, double start_time,
    double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, const double *regions, std::size_t regions_length,
    const char *const *boundary_names, const std::uint8_t *boundary_kinds,
    const double *boundary_values, std::size_t boundary_count, int precision, char *summary,
    std::size_t summary_length, char *error, std::size_t error_length) {
  using namespace wasl_b200;
  return twin(summary, summary_length, error, error_length, [&] {
    // bridge.cpp:183-216
    constexpr std::size_t width = 10;
    if (regions_length % width != 0 || (regions_length && !regions))
      throw std::runtime_error("initial.regions: invalid Euler region data");
    wasl::EulerCase c;
    c.files = case_files(mesh_path, output_path, restart_path);
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
    for (std::size_t i = 0; i < regions_length; i += width) {
      const double *r = regions + i;
      const int shape = static_cast<int>(r[0]);
      if (shape < 0 || shape > 2)
        throw std::runtime_error("initial.regions: invalid Euler region shape");
      wasl::EulerRegion region;
      region.shape = static_cast<wasl::EulerRegion::Shape>(shape);
      region.lower = r[1];
      region.upper = r[2];
      region.center_x = r[3];
      region.center_y = r[4];
      region.radius = r[5];
      region.value = {r[6], r[7], r[8], r[9]};
      c.initial_regions.push_back(region);
    }
    c.boundaries = named_boundaries(boundary_names, boundary_kinds, boundary_values,
                                    boundary_count);
    return summary_message(run_euler_case_gpu(c, precision));
  });
}

extern "C" int wasl_run_euler_case_gpu(
    const char *mesh_path, const char *output_path, const char *restart_path, int limiting,
    double sensor_threshold, double density_floor, double pressure_floor, int dimensions,
    int polynomial_order, double heat_capacity_ratio, double cfl, double start_time,
    double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, const double *regions, std::size_t regions_length,
    const char *const *boundary_names, const std::uint8_t *boundary_kinds,
    const double *boundary_values, std::size_t boundary_count, char *summary,
    std::size_t summary_length, char *error, std::size_t error_length) {
  return wasl_run_euler_case_gpu_ex(
      mesh_path, output_path, restart_path, limiting, sensor_threshold, density_floor,
      pressure_floor, dimensions, polynomial_order, heat_capacity_ratio, cfl, start_time, end_time,
      max_steps, history_interval, visualization_interval, checkpoint_interval, keep_checkpoints,
      regions, regions_length, boundary_names, boundary_kinds, boundary_values, boundary_count,
      WASL_PLAIN_FP64, summary, summary_length, error, error_length);
}

extern "C" int wasl_run_scalar_advection_case_gpu(
    const char *mesh_path, const char *output_path, const char *restart_path, int mpi,
    int dimensions, int polynomial_order, double velocity_x, double velocity_y, double cfl,
    double start_time, double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, double initial_default, int initial_sine,
    double initial_sine_amplitude, const double *intervals, std::size_t intervals_length,
    const double *circles, std::size_t circles_length, const char *const *boundary_names,
    const std::uint8_t *boundary_kinds, const double *boundary_values,
    std::size_t boundary_count, char *summary, std::size_t summary_length, char *error,
    std::size_t error_length) {
  using namespace wasl_b200;
  return twin(summary, summary_length, error, error_length, [&] {
    // bridge.cpp:141-181
    if (intervals_length % 3 != 0 || (intervals_length && !intervals))
      throw std::runtime_error("initial.regions: invalid interval data");
    if (circles_length % 4 != 0 || (circles_length && !circles))
      throw std::runtime_error("initial.regions: invalid circle data");
    wasl::ScalarAdvectionCase c;
    c.files = case_files(mesh_path, output_path, restart_path);
    c.run = {start_time,           end_time,           max_steps,       history_interval,
             visualization_interval, checkpoint_interval, keep_checkpoints};
    c.mpi = mpi != 0;
    c.dimensions = dimensions;
    c.polynomial_order = polynomial_order;
    c.wavespeed = velocity_x;
    c.velocity_y = velocity_y;
    c.cfl = cfl;
    c.initial_default = initial_default;
    c.initial_sine = initial_sine != 0;
    c.initial_sine_amplitude = initial_sine_amplitude;
    for (std::size_t i = 0; i < intervals_length; i += 3)
      c.initial_intervals.push_back({intervals[i], intervals[i + 1], intervals[i + 2]});
    for (std::size_t i = 0; i < circles_length; i += 4)
      c.initial_circles.push_back({circles[i], circles[i + 1], circles[i + 2], circles[i + 3]});
    c.boundaries = named_boundaries(boundary_names, boundary_kinds, boundary_values,
                                    boundary_count);
    return summary_message(run_scalar_advection_case_gpu(c));
  });
}

extern "C" int wasl_inspect_checkpoint(const char *checkpoint_path, char *summary,
                                       std::size_t summary_length, char *error,
                                       std::size_t error_length) {
  using namespace wasl_b200;
  return twin(summary, summary_length, error, error_length, [&] {
    // bridge.cpp:93-101
    const auto checkpoint = wasl::read_checkpoint(checkpoint_path ? checkpoint_path : "");
    std::ostringstream out;
    out.precision(17);
    out << "step=" << checkpoint.step << " time=" << checkpoint.time
        << " variables=" << checkpoint.variable_count << " modes=" << checkpoint.mode_count
        << " elements=" << checkpoint.element_count;
    return out.str();
  });
}

extern "C" int wasl_inspect_prepared_mesh(const char *mesh_path, char *summary,
                                          std::size_t summary_length, char *error,
                                          std::size_t error_length) {
  using namespace wasl_b200;
  return twin(summary, summary_length, error, error_length, [&] {
    // bridge.cpp:103-107
    const auto mesh = wasl::read_prepared_mesh(mesh_path ? mesh_path : "");
    return std::to_string(mesh.dimension) + "D mesh with " + std::to_string(mesh.element_count()) +
           " elements";
  });
}

extern "C" int wasl_export_checkpoint(const char *checkpoint_path, const char *mesh_path,
                                      const char *output_path, char *summary,
                                      std::size_t summary_length, char *error,
                                      std::size_t error_length) {
  using namespace wasl_b200;
  return twin(summary, summary_length, error, error_length, [&] {
    // bridge.cpp:109-129: cell averages c_0 / sqrt(2) of every variable to VTU.
    const auto checkpoint = wasl::read_checkpoint(checkpoint_path ? checkpoint_path : "");
    const auto mesh = wasl::read_prepared_mesh(mesh_path ? mesh_path : "");
    if (checkpoint.element_count != mesh.element_count())
      throw std::runtime_error("checkpoint export: mesh element count mismatch");
    const double inverse_sqrt2 = 1.0 / std::sqrt(2.0);
    const std::size_t nv = checkpoint.variable_count, ne = checkpoint.element_count;
    std::vector<double> averages(nv * ne);
    for (std::size_t v = 0; v < nv; ++v)
      for (std::size_t e = 0; e < ne; ++e)
        averages[e * nv + v] = checkpoint.coefficients[(v * checkpoint.mode_count) * ne + e] *
                               inverse_sqrt2;
    wasl::write_vtu(output_path ? output_path : "", mesh, averages, nv);
    return "exported " + std::to_string(ne) + " cells";
  });
}

extern "C" int wasl_prepare_mesh(const char *source_path, const char *output_path, char *summary,
                                 std::size_t summary_length, char *error,
                                 std::size_t error_length) {
  using namespace wasl_b200;
  return twin(summary, summary_length, error, error_length, [&] {
    // bridge.cpp:79-91
    const auto document = wasl::read_msh(source_path ? source_path : "");
    const bool has_triangles = std::any_of(
        document.elements.begin(), document.elements.end(),
        [](const auto &element) { return element.element_type == wasl::msh_triangle_element; });
    const auto prepared = has_triangles ? wasl::prepare_mesh(wasl::build_triangle_mesh(document))
                                        : wasl::prepare_mesh(wasl::build_line_mesh(document));
    wasl::write_prepared_mesh(output_path ? output_path : "", prepared);
    return "prepared " + std::to_string(prepared.element_count()) + " elements";
  });
}

extern "C" int wasl_prepare_mpi_run_directory(const char *root_path, const char *effective_config,
                                              char *summary, std::size_t summary_length,
                                              char *error, std::size_t error_length) {
  using namespace wasl_b200;
  return twin(summary, summary_length, error, error_length, [&] {
    // bridge.cpp:131-133
    return wasl::prepare_mpi_run_directory(root_path ? root_path : "",
                                           effective_config ? effective_config : "")
        .string();
  });
}
