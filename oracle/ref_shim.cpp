// ref_shim.cpp -- flat C entry points over the reference solver's own C++ code.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the reference numerical
// core from its sources (which stay where they are) together with this file
// into oracle/_ref/libwaslref.so.  The tests call it to pin the C restatement
// in wasl_oracle.c against the reference itself; nothing in the product links
// it.  Every wr_* function mirrors the wo_* function of the same name.
//
// It also supplies stand-ins for the four HDF5 functions the case layer links
// (cpp/src/io/checkpoint_file.cpp, cpp/src/io/prepared_mesh_file.cpp), in a
// plain binary format, because HDF5 is not installed here.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "wasl/boundaries/line_boundary_conditions.hpp"
#include "wasl/case/euler_case.hpp"
#include "wasl/case/scalar_advection_case.hpp"
#include "wasl/mesh/prepared/prepare_mesh.hpp"
#include "wasl/boundaries/line_euler_exterior.hpp"
#include "wasl/boundaries/periodic_triangle_trace.hpp"
#include "wasl/dg/euler/line_residual.hpp"
#include "wasl/dg/euler/triangle_residual.hpp"
#include "wasl/dg/scalar_advection/line_residual.hpp"
#include "wasl/dg/scalar_advection/triangle_residual.hpp"
#include "wasl/flux/hllc.hpp"
#include "wasl/io/checkpoint_file.hpp"
#include "wasl/io/prepared_mesh_file.hpp"
#include "wasl/limiting/euler_limiter_stencil.hpp"
#include "wasl/limiting/euler_modal_limiter.hpp"
#include "wasl/limiting/troubled_cell/modal_decay.hpp"
#include "wasl/mesh/line/build_line_mesh.hpp"
#include "wasl/mesh/msh/msh_document.hpp"
#include "wasl/mesh/triangle/build_triangle_mesh.hpp"
#include "wasl/time/cfl_timestep.hpp"
#include "wasl/time/line_advection_step.hpp"
#include "wasl/time/ssp_rk3.hpp"

namespace {

thread_local std::string last_error;

template <typename F> int guarded(F &&body) {
  try {
    body();
    return 0;
  } catch (const std::exception &error) {
    last_error = error.what();
    return -1;
  }
}

struct TriHandle {
  wasl::TriangleMesh mesh;
};
struct LineHandle {
  wasl::LineMesh mesh;
};
struct StencilHandle {
  wasl::EulerLimiterStencil stencil;
};

// ---- binary stand-ins for the HDF5 files ----------------------------------

template <typename T> void put(std::ofstream &out, const T &value) {
  out.write(reinterpret_cast<const char *>(&value), sizeof(T));
}
template <typename T> void put_vector(std::ofstream &out, const std::vector<T> &values) {
  put<std::uint64_t>(out, values.size());
  out.write(reinterpret_cast<const char *>(values.data()),
            static_cast<std::streamsize>(values.size() * sizeof(T)));
}
template <typename T> T get(std::ifstream &in) {
  T value{};
  in.read(reinterpret_cast<char *>(&value), sizeof(T));
  return value;
}
template <typename T> std::vector<T> get_vector(std::ifstream &in) {
  std::vector<T> values(get<std::uint64_t>(in));
  in.read(reinterpret_cast<char *>(values.data()),
          static_cast<std::streamsize>(values.size() * sizeof(T)));
  return values;
}

} // namespace

namespace wasl {

void write_checkpoint(const std::filesystem::path &path, const Checkpoint &checkpoint) {
  validate_checkpoint(checkpoint);
  if (path.has_parent_path())
    std::filesystem::create_directories(path.parent_path());
  std::ofstream out(path, std::ios::binary | std::ios::trunc);
  put(out, checkpoint.time);
  put(out, checkpoint.step);
  put(out, checkpoint.variable_count);
  put(out, checkpoint.mode_count);
  put(out, checkpoint.element_count);
  put_vector(out, std::vector<char>(checkpoint.prepared_mesh.begin(), checkpoint.prepared_mesh.end()));
  put_vector(out, checkpoint.coefficients);
  put(out, checkpoint.partition_rank);
  put(out, checkpoint.partition_rank_count);
  put(out, checkpoint_global_element_count(checkpoint));
  put_vector(out, checkpoint_element_indices(checkpoint));
}

Checkpoint read_checkpoint(const std::filesystem::path &path) {
  if (!std::filesystem::is_regular_file(path))
    throw std::runtime_error("checkpoint read: file does not exist: " + path.string());
  std::ifstream in(path, std::ios::binary);
  Checkpoint checkpoint;
  checkpoint.time = get<double>(in);
  checkpoint.step = get<std::uint64_t>(in);
  checkpoint.variable_count = get<std::uint64_t>(in);
  checkpoint.mode_count = get<std::uint64_t>(in);
  checkpoint.element_count = get<std::uint64_t>(in);
  const auto mesh = get_vector<char>(in);
  checkpoint.prepared_mesh.assign(mesh.begin(), mesh.end());
  checkpoint.coefficients = get_vector<double>(in);
  checkpoint.partition_rank = get<int>(in);
  checkpoint.partition_rank_count = get<int>(in);
  checkpoint.global_element_count = get<std::uint64_t>(in);
  checkpoint.element_indices = get_vector<std::int64_t>(in);
  validate_checkpoint(checkpoint);
  return checkpoint;
}

void write_prepared_mesh(const std::filesystem::path &path, const PreparedMesh &m) {
  if (path.has_parent_path())
    std::filesystem::create_directories(path.parent_path());
  std::ofstream out(path, std::ios::binary | std::ios::trunc);
  put(out, m.dimension);
  put(out, m.nodes_per_element);
  put_vector(out, m.node_tags);
  put_vector(out, m.points);
  put_vector(out, m.element_nodes);
  put_vector(out, m.element_physical_tags);
  put_vector(out, m.element_metrics);
  put_vector(out, m.face_nodes);
  put_vector(out, m.face_elements);
  put_vector(out, m.face_local_edges);
  put_vector(out, m.face_normals);
  put_vector(out, m.face_measures);
  put_vector(out, m.face_physical_tags);
  put_vector(out, m.physical_name_dimensions);
  put_vector(out, m.physical_name_tags);
  put_vector(out, m.physical_name_offsets);
  put_vector(out, m.physical_name_bytes);
  put(out, m.partition_rank_count);
  put_vector(out, m.element_owners);
  put_vector(out, m.face_owners);
}

PreparedMesh read_prepared_mesh(const std::filesystem::path &path) {
  if (!std::filesystem::is_regular_file(path))
    throw std::runtime_error("prepared mesh read: file does not exist: " + path.string());
  std::ifstream in(path, std::ios::binary);
  PreparedMesh m;
  m.dimension = get<int>(in);
  m.nodes_per_element = get<int>(in);
  m.node_tags = get_vector<std::int64_t>(in);
  m.points = get_vector<double>(in);
  m.element_nodes = get_vector<std::int64_t>(in);
  m.element_physical_tags = get_vector<std::int32_t>(in);
  m.element_metrics = get_vector<double>(in);
  m.face_nodes = get_vector<std::int64_t>(in);
  m.face_elements = get_vector<std::int32_t>(in);
  m.face_local_edges = get_vector<std::int32_t>(in);
  m.face_normals = get_vector<double>(in);
  m.face_measures = get_vector<double>(in);
  m.face_physical_tags = get_vector<std::int32_t>(in);
  m.physical_name_dimensions = get_vector<std::int32_t>(in);
  m.physical_name_tags = get_vector<std::int32_t>(in);
  m.physical_name_offsets = get_vector<std::uint64_t>(in);
  m.physical_name_bytes = get_vector<unsigned char>(in);
  m.partition_rank_count = get<int>(in);
  m.element_owners = get_vector<std::int32_t>(in);
  m.face_owners = get_vector<std::int32_t>(in);
  return m;
}

} // namespace wasl

extern "C" {

const char *wr_last_error() { return last_error.c_str(); }

// ---- meshes ----------------------------------------------------------------

// A document holding the nodes and triangles, with one surface entity so that
// build_triangle_mesh has the same input as the reference's in-code meshes.
void *wr_tri_mesh_new(std::int64_t node_count, const std::int64_t *tags, const double *xy,
                      std::int64_t element_count, const std::int64_t *element_nodes) {
  auto *handle = new TriHandle;
  const int rc = guarded([&] {
    wasl::MshDocument document;
    document.surface_entities.push_back({1, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, {1}, {}});
    for (std::int64_t i = 0; i < node_count; ++i)
      document.nodes.push_back({tags[i], 2, 1, xy[2 * i], xy[2 * i + 1], 0.0});
    for (std::int64_t e = 0; e < element_count; ++e)
      document.elements.push_back({e + 1, 2, 1, wasl::msh_triangle_element,
                                   {element_nodes[3 * e], element_nodes[3 * e + 1],
                                    element_nodes[3 * e + 2]}});
    handle->mesh = wasl::build_triangle_mesh(document);
  });
  if (rc != 0) {
    delete handle;
    return nullptr;
  }
  return handle;
}

void wr_tri_mesh_free(void *handle) { delete static_cast<TriHandle *>(handle); }

std::int64_t wr_tri_mesh_face_count(void *handle) {
  return static_cast<std::int64_t>(static_cast<TriHandle *>(handle)->mesh.faces.size());
}

void wr_tri_mesh_export(void *handle, double *vertices, std::int64_t *nodes, std::int32_t *left,
                        std::int32_t *right, std::int32_t *left_edge, std::int32_t *right_edge,
                        std::int64_t *left_v0, std::int64_t *right_v0, double *nx, double *ny) {
  const auto &mesh = static_cast<TriHandle *>(handle)->mesh;
  for (std::size_t e = 0; e < mesh.elements.size(); ++e) {
    const auto &el = mesh.elements[e];
    const double v[6] = {el.x0, el.y0, el.x1, el.y1, el.x2, el.y2};
    std::memcpy(vertices + 6 * e, v, sizeof(v));
    nodes[3 * e] = el.node0;
    nodes[3 * e + 1] = el.node1;
    nodes[3 * e + 2] = el.node2;
  }
  for (std::size_t f = 0; f < mesh.faces.size(); ++f) {
    const auto &face = mesh.faces[f];
    left[f] = face.left_element;
    right[f] = face.right_element;
    left_edge[f] = face.left_local_edge;
    right_edge[f] = face.right_local_edge;
    left_v0[f] = face.left_vertex0;
    right_v0[f] = face.right_vertex0;
    nx[f] = face.outward_normal_x;
    ny[f] = face.outward_normal_y;
  }
}

void *wr_line_mesh_new(std::int64_t node_count, const std::int64_t *tags, const double *x,
                       std::int64_t element_count, const std::int64_t *element_nodes) {
  auto *handle = new LineHandle;
  const int rc = guarded([&] {
    wasl::MshDocument document;
    document.point_entities.push_back({1, 0.0, 0.0, 0.0, {}});
    document.curve_entities.push_back({1, 0, 0, 0, 1, 0, 0, {1}, {}});
    for (std::int64_t i = 0; i < node_count; ++i)
      document.nodes.push_back({tags[i], 1, 1, x[i], 0.0, 0.0});
    for (std::int64_t e = 0; e < element_count; ++e)
      document.elements.push_back({e + 1, 1, 1, wasl::msh_line_element,
                                   {element_nodes[2 * e], element_nodes[2 * e + 1]}});
    handle->mesh = wasl::build_line_mesh(document);
  });
  if (rc != 0) {
    delete handle;
    return nullptr;
  }
  return handle;
}

void wr_line_mesh_free(void *handle) { delete static_cast<LineHandle *>(handle); }

void wr_line_mesh_export(void *handle, double *x_left, double *x_right) {
  const auto &mesh = static_cast<LineHandle *>(handle)->mesh;
  for (std::size_t e = 0; e < mesh.elements.size(); ++e) {
    x_left[e] = mesh.elements[e].x_left;
    x_right[e] = mesh.elements[e].x_right;
  }
}

// ---- residuals -------------------------------------------------------------

void wr_euler_tri_residual(void *handle, double gamma, int p, const double *c, const double *ext,
                           double *rhs) {
  wasl::euler_triangle_residual(static_cast<TriHandle *>(handle)->mesh, wasl::Euler{gamma},
                                wasl::hllc_flux, p, c, ext, rhs);
}

void wr_euler_line_residual(void *handle, double gamma, int p, const double *c, const double *ext,
                            double *rhs) {
  wasl::euler_line_residual(static_cast<LineHandle *>(handle)->mesh, wasl::Euler{gamma},
                            wasl::hllc_flux, p, c, ext, rhs);
}

void wr_scalar_line_residual(void *handle, double a, int p, const double *c, const double *ext,
                             double *rhs) {
  wasl::scalar_advection_residual(static_cast<LineHandle *>(handle)->mesh,
                                  wasl::ScalarAdvection{a}, p, c, ext, rhs);
}

void wr_scalar_tri_residual(void *handle, double vx, double vy, int p, const double *c,
                            const double *ext, double *rhs) {
  wasl::triangle_scalar_advection_residual(static_cast<TriHandle *>(handle)->mesh,
                                           wasl::ScalarAdvection2D{vx, vy}, p, c, ext, rhs);
}

void wr_hllc_flux(double gamma, const double *l, const double *r, double nx, double ny,
                  double *flux) {
  const auto f = wasl::hllc_flux(wasl::Euler{gamma}, {l[0], l[1], l[2], l[3]},
                                 {r[0], r[1], r[2], r[3]}, nx, ny);
  flux[0] = f.density;
  flux[1] = f.momentum_x;
  flux[2] = f.momentum_y;
  flux[3] = f.total_energy;
}

// ---- exterior traces ---------------------------------------------------------

int wr_periodic_tri_trace(void *handle, int p, std::int32_t *donors, double *basis) {
  return guarded([&] {
    const auto trace = wasl::periodic_triangle_trace(static_cast<TriHandle *>(handle)->mesh, p);
    std::memcpy(donors, trace.elements.data(), trace.elements.size() * sizeof(std::int32_t));
    std::memcpy(basis, trace.basis.data(), trace.basis.size() * sizeof(double));
  });
}

void wr_periodic_tri_euler_exterior(void *handle, int p, const std::int32_t *donors,
                                    const double *basis, const double *c, double *ext) {
  const auto &mesh = static_cast<TriHandle *>(handle)->mesh;
  const std::size_t M = wasl::triangle_mode_count(p), Q = p + 1, F = mesh.faces.size();
  wasl::PeriodicTriangleTrace trace;
  trace.elements.assign(donors, donors + F * Q);
  trace.basis.assign(basis, basis + F * Q * M);
  trace.point_count = static_cast<int>(Q);
  const std::size_t ne = mesh.num_elements();
  const std::vector<double> state(c, c + 4 * M * ne);
  const auto out = wasl::periodic_triangle_euler_exterior(trace, state, ne, M, F);
  std::memcpy(ext, out.data(), out.size() * sizeof(double));
}

int wr_line_euler_exterior(void *handle, int p, int left_kind, int right_kind, const double *c,
                           double *ext) {
  return guarded([&] {
    const auto &mesh = static_cast<LineHandle *>(handle)->mesh;
    wasl::LineBoundaryConditions conditions;
    conditions.left.kind = static_cast<wasl::BoundaryKind>(left_kind);
    conditions.right.kind = static_cast<wasl::BoundaryKind>(right_kind);
    const std::size_t n = 4 * wasl::line_mode_count(p) * mesh.num_elements();
    const auto out = wasl::line_euler_exterior(mesh, p, conditions, std::vector<double>(c, c + n));
    std::memcpy(ext, out.data(), out.size() * sizeof(double));
  });
}

// ---- limiter -------------------------------------------------------------------

void *wr_tri_stencil_new(void *handle, int p, const std::int32_t *donors) {
  auto *s = new StencilHandle;
  const auto &mesh = static_cast<TriHandle *>(handle)->mesh;
  std::vector<std::int32_t> periodic;
  if (donors)
    periodic.assign(donors, donors + mesh.faces.size() * static_cast<std::size_t>(p + 1));
  s->stencil = wasl::make_euler_limiter_stencil(mesh, p, periodic, p + 1);
  return s;
}

void *wr_line_stencil_new(void *handle, int p, int periodic) {
  auto *s = new StencilHandle;
  s->stencil = wasl::make_euler_limiter_stencil(
      static_cast<LineHandle *>(handle)->mesh, p,
      periodic ? wasl::LineEnds::periodic : wasl::LineEnds::open);
  return s;
}

void wr_stencil_free(void *s) { delete static_cast<StencilHandle *>(s); }

void wr_stencil_export(void *s, std::int32_t *neighbors, double *transforms, double *nx,
                       double *ny, double *check, int *check_count) {
  const auto &st = static_cast<StencilHandle *>(s)->stencil;
  std::memcpy(neighbors, st.neighbors.data(), st.neighbors.size() * sizeof(std::int32_t));
  std::memcpy(transforms, st.transforms.data(), st.transforms.size() * sizeof(double));
  std::memcpy(nx, st.normal_x.data(), st.normal_x.size() * sizeof(double));
  std::memcpy(ny, st.normal_y.data(), st.normal_y.size() * sizeof(double));
  std::memcpy(check, st.check_basis.data(), st.check_basis.size() * sizeof(double));
  *check_count = static_cast<int>(st.check_point_count());
}

int wr_limit_euler(void *s, double gamma, double threshold, double rf, double pf, double *c) {
  return guarded([&] {
    const auto &st = static_cast<StencilHandle *>(s)->stencil;
    const std::size_t n = 4 * st.mode_count * st.element_count;
    std::vector<double> state(c, c + n);
    wasl::limit_euler_modal(st, wasl::Euler{gamma}, threshold, rf, pf, state);
    std::memcpy(c, state.data(), n * sizeof(double));
  });
}

// ---- time step -------------------------------------------------------------------

int wr_euler_tri_cfl(void *handle, double gamma, const double *c, int p, double cfl, double *dt) {
  return guarded([&] {
    const auto &mesh = static_cast<TriHandle *>(handle)->mesh;
    const std::size_t M = wasl::triangle_mode_count(p);
    *dt = wasl::euler_cfl_timestep(mesh, wasl::Euler{gamma},
                                   std::vector<double>(c, c + 4 * M * mesh.num_elements()), M, p,
                                   cfl);
  });
}

int wr_euler_line_cfl(void *handle, double gamma, const double *c, int p, double cfl, double *dt) {
  return guarded([&] {
    const auto &mesh = static_cast<LineHandle *>(handle)->mesh;
    const std::size_t M = wasl::line_mode_count(p);
    *dt = wasl::euler_cfl_timestep(mesh, wasl::Euler{gamma},
                                   std::vector<double>(c, c + 4 * M * mesh.num_elements()), M, p,
                                   cfl);
  });
}

// One SSP-RK3 step of 2D Euler with the periodic exterior, as the case driver
// composes it (cpp/src/case/euler_triangle.cpp:26-49).  stencil may be null.
int wr_euler_tri_step(void *handle, const std::int32_t *donors, const double *basis, void *stencil,
                      double threshold, double rf, double pf, double gamma, int p, double dt,
                      double *c) {
  return guarded([&] {
    const auto &mesh = static_cast<TriHandle *>(handle)->mesh;
    const std::size_t M = wasl::triangle_mode_count(p), Q = p + 1, F = mesh.faces.size();
    const std::size_t ne = mesh.num_elements();
    wasl::PeriodicTriangleTrace trace;
    trace.elements.assign(donors, donors + F * Q);
    trace.basis.assign(basis, basis + F * Q * M);
    trace.point_count = static_cast<int>(Q);
    const wasl::Euler equation{gamma};
    const wasl::ResidualFunction residual = [&](std::vector<double> &stage,
                                                std::vector<double> &rhs) {
      const auto exterior = wasl::periodic_triangle_euler_exterior(trace, stage, ne, M, F);
      wasl::euler_triangle_residual(mesh, equation, wasl::hllc_flux, p, stage.data(),
                                    exterior.data(), rhs.data());
    };
    const wasl::StateFunction limit = [&](std::vector<double> &state) {
      if (stencil)
        wasl::limit_euler_modal(static_cast<StencilHandle *>(stencil)->stencil, equation,
                                threshold, rf, pf, state);
    };
    std::vector<double> state(c, c + 4 * M * ne);
    wasl::SspRk3Workspace workspace;
    wasl::ssp_rk3_step(dt, residual, limit, state, workspace);
    std::memcpy(c, state.data(), state.size() * sizeof(double));
  });
}

// wr_euler_tri_step with a choice of exterior and the troubled-cell flag set
// of each stage.  boundary_kind 0: the periodic exterior from donors/basis;
// 3: the owner's own trace at every boundary edge point (the harness's 2D
// transmissive boundary; the reference's 2D cases are periodic only), built
// with the reference's edge rules, basis and evaluate_euler_state, so it is
// the left trace the residual itself evaluates.  flags [3][ne] (may be null):
// per stage, the sensor verdict the limiter reaches on each element, from the
// reference's modal_energy on the stage state it receives
// (cpp/src/limiting/euler_modal_limiter.cpp:18-24).
int wr_euler_tri_step_ex(void *handle, int boundary_kind, const std::int32_t *donors,
                         const double *basis, void *stencil, double threshold, double rf,
                         double pf, double gamma, int p, double dt, double *c,
                         std::uint8_t *flags) {
  return guarded([&] {
    const auto &mesh = static_cast<TriHandle *>(handle)->mesh;
    const std::size_t M = wasl::triangle_mode_count(p), Q = p + 1, F = mesh.faces.size();
    const std::size_t ne = mesh.num_elements();
    const wasl::ModalLayout layout{M, ne};
    wasl::PeriodicTriangleTrace trace;
    if (boundary_kind == 0) {
      trace.elements.assign(donors, donors + F * Q);
      trace.basis.assign(basis, basis + F * Q * M);
      trace.point_count = static_cast<int>(Q);
    } else if (boundary_kind != 3) {
      throw std::invalid_argument("boundary kind must be 0 (periodic) or 3 (transmissive)");
    }
    const auto edge_rules = wasl::triangle_edge_rules(p);
    std::vector<double> edge_basis(M);
    const wasl::Euler equation{gamma};
    const wasl::ResidualFunction residual = [&](std::vector<double> &stage,
                                                std::vector<double> &rhs) {
      std::vector<double> exterior;
      if (boundary_kind == 0) {
        exterior = wasl::periodic_triangle_euler_exterior(trace, stage, ne, M, F);
      } else {
        exterior.assign(4 * F * Q, 0.0);
        for (std::size_t f = 0; f < F; ++f) {
          const auto &face = mesh.faces[f];
          if (!face.is_boundary())
            continue;
          const auto &rule = edge_rules[static_cast<std::size_t>(face.left_local_edge)];
          for (std::size_t q = 0; q < Q; ++q) {
            wasl::dubiner_basis(rule.xi[q], rule.eta[q], p, edge_basis.data());
            const wasl::EulerConserved s = wasl::evaluate_euler_state(
                layout, stage.data(), static_cast<std::size_t>(face.left_element),
                edge_basis.data());
            for (int v = 0; v < 4; ++v)
              exterior[(static_cast<std::size_t>(v) * F + f) * Q + q] = wasl::euler_component(s, v);
          }
        }
      }
      wasl::euler_triangle_residual(mesh, equation, wasl::hllc_flux, p, stage.data(),
                                    exterior.data(), rhs.data());
    };
    int stage_index = 0;
    const wasl::StateFunction limit = [&](std::vector<double> &state) {
      if (!stencil)
        return;
      const auto &st = static_cast<StencilHandle *>(stencil)->stencil;
      if (flags) {
        std::uint8_t *out = flags + static_cast<std::size_t>(stage_index) * ne;
        for (std::size_t e = 0; e < ne; ++e) {
          const auto energy = wasl::modal_energy(state.data() + layout.index(0, 0, e), ne,
                                                 st.mode_count, st.highest_degree_begin);
          out[e] = st.polynomial_order > 0 &&
                           !(energy.total == 0.0 || energy.highest_degree / energy.total <= threshold)
                       ? 1
                       : 0;
        }
      }
      ++stage_index;
      wasl::limit_euler_modal(st, equation, threshold, rf, pf, state);
    };
    std::vector<double> state(c, c + 4 * M * ne);
    wasl::SspRk3Workspace workspace;
    wasl::ssp_rk3_step(dt, residual, limit, state, workspace);
    std::memcpy(c, state.data(), state.size() * sizeof(double));
  });
}

int wr_euler_line_step(void *handle, int left_kind, int right_kind, void *stencil,
                       double threshold, double rf, double pf, double gamma, int p, double dt,
                       double *c) {
  return guarded([&] {
    const auto &mesh = static_cast<LineHandle *>(handle)->mesh;
    const std::size_t M = wasl::line_mode_count(p), ne = mesh.num_elements();
    wasl::LineBoundaryConditions conditions;
    conditions.left.kind = static_cast<wasl::BoundaryKind>(left_kind);
    conditions.right.kind = static_cast<wasl::BoundaryKind>(right_kind);
    const wasl::Euler equation{gamma};
    const wasl::ResidualFunction residual = [&](std::vector<double> &stage,
                                                std::vector<double> &rhs) {
      const auto exterior = wasl::line_euler_exterior(mesh, p, conditions, stage);
      wasl::euler_line_residual(mesh, equation, wasl::hllc_flux, p, stage.data(),
                                exterior.data(), rhs.data());
    };
    const wasl::StateFunction limit = [&](std::vector<double> &state) {
      if (stencil)
        wasl::limit_euler_modal(static_cast<StencilHandle *>(stencil)->stencil, equation,
                                threshold, rf, pf, state);
    };
    std::vector<double> state(c, c + 4 * M * ne);
    wasl::SspRk3Workspace workspace;
    wasl::ssp_rk3_step(dt, residual, limit, state, workspace);
    std::memcpy(c, state.data(), state.size() * sizeof(double));
  });
}

void wr_scalar_line_step(void *handle, int left_kind, double left_value, int right_kind,
                         double right_value, double a, int p, double dt, double *c) {
  const auto &mesh = static_cast<LineHandle *>(handle)->mesh;
  const wasl::LineBoundaryConditions conditions{
      {static_cast<wasl::BoundaryKind>(left_kind), left_value},
      {static_cast<wasl::BoundaryKind>(right_kind), right_value}};
  const auto exterior = wasl::make_line_boundary_exterior(mesh, p, conditions);
  std::vector<double> state(c, c + wasl::line_mode_count(p) * mesh.num_elements());
  wasl::SspRk3Workspace workspace;
  wasl::ssp_rk3_step(mesh, wasl::ScalarAdvection{a}, p, dt, exterior, state, workspace);
  std::memcpy(c, state.data(), state.size() * sizeof(double));
}

// The serial run of a periodic 1D advection case, as
// cpp/src/case/scalar_advection_line.cpp:11-33 composes it (CFL step fixed at
// setup, SSP-RK3 with the reused workspace) inside the run loop's time
// arithmetic (cpp/src/case/serial_case_runner.cpp:107-142), without the
// files: the reference's CPU run of the 400-cell configuration, timed whole.
// c: the solver layout U[element][mode]; returns -1 if time cannot advance.
int wr_scalar_line_run(void *handle, int p, double a, double cfl, double start_time,
                       double end_time, std::uint64_t max_steps, double *c,
                       std::uint64_t *steps, double *time) {
  return guarded([&] {
    const auto &mesh = static_cast<LineHandle *>(handle)->mesh;
    const wasl::ScalarAdvection equation{a};
    const auto exterior = wasl::make_line_boundary_exterior(mesh, p, {});
    const double cfl_step = wasl::advection_cfl_timestep(mesh, equation, p, cfl);
    std::vector<double> state(c, c + wasl::line_mode_count(p) * mesh.num_elements());
    wasl::SspRk3Workspace workspace;
    double t = start_time;
    std::uint64_t n = 0;
    while (t < end_time && n < max_steps) {
      const double remaining = end_time - t;
      const double dt = std::min(cfl_step > 0.0 ? cfl_step : remaining, remaining);
      if (dt <= 0.0 || t + dt == t)
        throw std::runtime_error("simulation: timestep cannot advance time");
      wasl::ssp_rk3_step(mesh, equation, p, dt, exterior, state, workspace);
      t += dt;
      ++n;
    }
    std::memcpy(c, state.data(), state.size() * sizeof(double));
    *steps = n;
    *time = t;
  });
}

// ---- whole cases through the reference's own run loop ------------------------

int wr_write_prepared_tri_mesh(void *handle, const char *path) {
  return guarded([&] {
    wasl::write_prepared_mesh(path, wasl::prepare_mesh(static_cast<TriHandle *>(handle)->mesh));
  });
}

int wr_write_prepared_line_mesh(void *handle, const char *path) {
  return guarded([&] {
    wasl::write_prepared_mesh(path, wasl::prepare_mesh(static_cast<LineHandle *>(handle)->mesh));
  });
}

// ---- the bridge's coarse functions from C arguments ----------------------------
//
// crates/wasl-bridge/src/bridge.cpp:79-216 with rust::Str -> const char *,
// rust::Slice<T> -> (pointer, length) and the returned rust::String written to
// `summary`; its argument checks and messages are restated here, since the
// bridge itself needs the Rust toolchain's cxx headers.  The returned status
// is 0, or -1 with the message in wr_last_error().

void write_text(const std::string &text, char *out, std::size_t length) {
  if (out && length) {
    std::strncpy(out, text.c_str(), length - 1);
    out[length - 1] = '\0';
  }
}

std::string bridge_summary(const wasl::SimulationSummary &summary) {
  std::ostringstream message;
  message.precision(17);
  message << "step=" << summary.step << " time=" << summary.time
          << " checkpoint=" << summary.checkpoint.string();
  return message.str();
}

std::vector<wasl::NamedBoundary> bridge_boundaries(const char *const *names,
                                                   const std::uint8_t *kinds,
                                                   const double *values, std::size_t count) {
  std::vector<wasl::NamedBoundary> boundaries;
  for (std::size_t i = 0; i < count; ++i) {
    if (kinds[i] > static_cast<std::uint8_t>(wasl::BoundaryKind::outflow))
      throw std::runtime_error("boundaries: invalid boundary kind");
    boundaries.push_back({names[i], {static_cast<wasl::BoundaryKind>(kinds[i]), values[i]}});
  }
  return boundaries;
}

int wr_run_euler_case(const char *mesh_path, const char *output_path, const char *restart_path,
                      int limiting, double sensor_threshold, double density_floor,
                      double pressure_floor, int dimensions, int polynomial_order,
                      double heat_capacity_ratio, double cfl, double start_time, double end_time,
                      std::uint64_t max_steps, std::uint64_t history_interval,
                      std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
                      std::uint64_t keep_checkpoints, const double *regions,
                      std::size_t regions_length, const char *const *boundary_names,
                      const std::uint8_t *boundary_kinds, const double *boundary_values,
                      std::size_t boundary_count, char *summary, std::size_t summary_length) {
  return guarded([&] {
    constexpr std::size_t width = 10;
    if (regions_length % width != 0)
      throw std::runtime_error("initial.regions: invalid Euler region data");
    wasl::EulerCase c;
    c.files = {mesh_path, output_path, restart_path ? restart_path : ""};
    c.run = {start_time,           end_time,          max_steps,       history_interval,
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
    c.boundaries = bridge_boundaries(boundary_names, boundary_kinds, boundary_values,
                                     boundary_count);
    write_text(bridge_summary(wasl::run_euler_case(c)), summary, summary_length);
  });
}

int wr_run_scalar_advection_case(
    const char *mesh_path, const char *output_path, const char *restart_path, int mpi,
    int dimensions, int polynomial_order, double velocity_x, double velocity_y, double cfl,
    double start_time, double end_time, std::uint64_t max_steps, std::uint64_t history_interval,
    std::uint64_t visualization_interval, std::uint64_t checkpoint_interval,
    std::uint64_t keep_checkpoints, double initial_default, int initial_sine,
    double initial_sine_amplitude, const double *intervals, std::size_t intervals_length,
    const double *circles, std::size_t circles_length, const char *const *boundary_names,
    const std::uint8_t *boundary_kinds, const double *boundary_values,
    std::size_t boundary_count, char *summary, std::size_t summary_length) {
  return guarded([&] {
    if (intervals_length % 3 != 0)
      throw std::runtime_error("initial.regions: invalid interval data");
    if (circles_length % 4 != 0)
      throw std::runtime_error("initial.regions: invalid circle data");
    wasl::ScalarAdvectionCase c;
    c.files = {mesh_path, output_path, restart_path ? restart_path : ""};
    c.run = {start_time,           end_time,          max_steps,       history_interval,
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
    c.boundaries = bridge_boundaries(boundary_names, boundary_kinds, boundary_values,
                                     boundary_count);
    write_text(bridge_summary(wasl::run_scalar_advection_case(c)), summary, summary_length);
  });
}

int wr_inspect_checkpoint(const char *checkpoint_path, char *summary, std::size_t summary_length) {
  return guarded([&] {
    const auto checkpoint = wasl::read_checkpoint(checkpoint_path);
    std::ostringstream out;
    out.precision(17);
    out << "step=" << checkpoint.step << " time=" << checkpoint.time
        << " variables=" << checkpoint.variable_count << " modes=" << checkpoint.mode_count
        << " elements=" << checkpoint.element_count;
    write_text(out.str(), summary, summary_length);
  });
}

// A line mesh whose two end nodes carry the physical names "left" and
// "right" (point entities 1 and 2), so cases can name their end boundaries.
void *wr_line_mesh_named_new(std::int64_t node_count, const std::int64_t *tags, const double *x,
                             std::int64_t element_count, const std::int64_t *element_nodes) {
  auto *handle = new LineHandle;
  const int rc = guarded([&] {
    std::int64_t lo = 0, hi = 0;
    for (std::int64_t i = 1; i < node_count; ++i) {
      lo = x[i] < x[lo] ? i : lo;
      hi = x[i] > x[hi] ? i : hi;
    }
    wasl::MshDocument document;
    document.physical_names = {{0, 1, "left"}, {0, 2, "right"}};
    document.point_entities.push_back({1, x[lo], 0.0, 0.0, {1}});
    document.point_entities.push_back({2, x[hi], 0.0, 0.0, {2}});
    document.curve_entities.push_back({1, 0, 0, 0, 1, 0, 0, {}, {1, 2}});
    for (std::int64_t i = 0; i < node_count; ++i) {
      const int dim = i == lo || i == hi ? 0 : 1;
      const int entity = i == lo ? 1 : (i == hi ? 2 : 1);
      document.nodes.push_back({tags[i], dim, entity, x[i], 0.0, 0.0});
    }
    for (std::int64_t e = 0; e < element_count; ++e)
      document.elements.push_back({e + 1, 1, 1, wasl::msh_line_element,
                                   {element_nodes[2 * e], element_nodes[2 * e + 1]}});
    handle->mesh = wasl::build_line_mesh(document);
  });
  if (rc != 0) {
    delete handle;
    return nullptr;
  }
  return handle;
}

} // extern "C"
