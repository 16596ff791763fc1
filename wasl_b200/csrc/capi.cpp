// extern "C" entry points of libwasl_b200.so (declared in include/wasl_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>

#include "mesh.hpp"
#include "solver.hpp"

namespace wasl_b200 {
std::unique_ptr<Solver> make_euler_tri_solver(const wasl_gpu_config &cfg, TriTopology &&topo,
                                              const PartBoundary *part);
std::unique_ptr<Solver> make_scalar_tri_solver(const wasl_gpu_config &cfg, TriTopology &&topo,
                                               const PartBoundary *part);
std::unique_ptr<Solver> make_line_solver(const wasl_gpu_config &cfg, LineTopology &&topo);

bool form_supported(int precision, int dimensions, int equation, int p) {
  if (equation != WASL_EULER && equation != WASL_SCALAR_ADVECTION)
    return false;
  if (dimensions == 2 && equation == WASL_EULER)
    return (precision == WASL_PLAIN_FP64 && p >= 0 && p <= 3) ||
           (precision == WASL_MIXED && p >= 1 && p <= 3);
  if (dimensions == 2)
    return precision == WASL_PLAIN_FP64 && p >= 0 && p <= 3;
  if (dimensions == 1)
    return precision == WASL_PLAIN_FP64 && p >= 0 && p <= 6;
  return false;
}

std::unique_ptr<Solver> make_solver(const wasl_gpu_config &cfg, std::int64_t node_count,
                                    const std::int64_t *node_tags, const double *coordinates,
                                    std::int64_t element_count, const std::int64_t *element_nodes,
                                    const PartBoundary *part) {
  if (!form_supported(cfg.precision, cfg.dimensions, cfg.equation, cfg.polynomial_order))
    throw SolverError(WASL_ERR_ARGUMENT,
                      "unsupported combination of dimension, equation, order and precision");
  SetupTimes topology;
  topology.start();
  std::unique_ptr<Solver> solver;
  if (cfg.dimensions == 2) {
    TriTopology topo =
        build_triangle_topology(node_count, node_tags, coordinates, element_count, element_nodes);
    topology.lap(WASL_SETUP_TOPOLOGY);
    solver = cfg.equation == WASL_EULER ? make_euler_tri_solver(cfg, std::move(topo), part)
                                        : make_scalar_tri_solver(cfg, std::move(topo), part);
  } else {
    if (part)
      throw SolverError(WASL_ERR_ARGUMENT, "partition boundary: triangle meshes only");
    LineTopology topo =
        build_line_topology(node_count, node_tags, coordinates, element_count, element_nodes);
    topology.lap(WASL_SETUP_TOPOLOGY);
    solver = make_line_solver(cfg, std::move(topo));
  }
  solver->setup_times().ms[WASL_SETUP_TOPOLOGY] = topology.ms[WASL_SETUP_TOPOLOGY];
  return solver;
}
} // namespace wasl_b200

struct wasl_gpu {
  std::unique_ptr<wasl_b200::Solver> solver;
  std::string error;
};

namespace wasl_b200 {
// For the other C entry points built on a handle (halo.cu).
Solver *solver_of(wasl_gpu *handle) { return handle ? handle->solver.get() : nullptr; }
void set_handle_error(wasl_gpu *handle, const std::string &message) {
  if (handle)
    handle->error = message;
}
} // namespace wasl_b200

namespace {

template <typename F> int guarded(wasl_gpu *h, F &&body) {
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

void need(bool ok, const char *message) {
  if (!ok)
    throw wasl_b200::SolverError(WASL_ERR_ARGUMENT, message);
}

void copy_message(const std::string &message, char *error, size_t error_length) {
  if (error && error_length) {
    std::strncpy(error, message.c_str(), error_length - 1);
    error[error_length - 1] = '\0';
  }
}

// Checkpoint container: magic, format version 2, then the reference fields in
// declaration order (cpp/include/wasl/io/checkpoint.hpp:17-29).
constexpr char kMagic[8] = {'W', 'A', 'S', 'L', 'C', 'K', 'P', 'T'};

template <typename T> void put(std::ofstream &o, const T &v) {
  o.write(reinterpret_cast<const char *>(&v), sizeof(T));
}
template <typename T> T get(std::ifstream &i) {
  T v{};
  i.read(reinterpret_cast<char *>(&v), sizeof(T));
  if (!i)
    throw std::runtime_error("checkpoint read: truncated file");
  return v;
}

} // namespace

extern "C" {

void wasl_gpu_config_default(wasl_gpu_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->dimensions = 2;
  c->equation = WASL_EULER;
  c->polynomial_order = 2;
  c->heat_capacity_ratio = 1.4;
  c->boundary_left = c->boundary_right = WASL_PERIODIC;
  c->sensor_threshold = 1e-3;
  c->density_floor = 1e-10;
  c->pressure_floor = 1e-10;
  c->precision = WASL_PLAIN_FP64;
}

int wasl_gpu_form_supported(int precision, int dimensions, int equation, int p) {
  return wasl_b200::form_supported(precision, dimensions, equation, p) ? 1 : 0;
}

namespace {

int create_handle(const wasl_gpu_config *config, int64_t node_count, const int64_t *node_tags,
                  const double *node_coordinates, int64_t element_count,
                  const int64_t *element_nodes, const wasl_b200::PartBoundary *part,
                  wasl_gpu **handle, char *error, size_t error_length) {
  if (!handle || !config)
    return WASL_ERR_ARGUMENT;
  *handle = nullptr;
  auto h = std::make_unique<wasl_gpu>();
  const int rc = guarded(h.get(), [&] {
    need(node_count > 0 && element_count > 0, "mesh: empty node or element list");
    need(node_tags && node_coordinates && element_nodes, "mesh: null array");
    need(config->density_floor >= 0.0 && config->pressure_floor >= 0.0,
         "Euler positivity limiter: invalid modes or floors");
    h->solver = wasl_b200::make_solver(*config, node_count, node_tags, node_coordinates,
                                       element_count, element_nodes, part);
  });
  if (rc != WASL_OK) {
    copy_message(h->error, error, error_length);
    return rc;
  }
  *handle = h.release();
  return WASL_OK;
}

} // namespace

int wasl_gpu_create(const wasl_gpu_config *config, int64_t node_count, const int64_t *node_tags,
                    const double *node_coordinates, int64_t element_count,
                    const int64_t *element_nodes, wasl_gpu **handle, char *error,
                    size_t error_length) {
  return create_handle(config, node_count, node_tags, node_coordinates, element_count,
                       element_nodes, nullptr, handle, error, error_length);
}

int wasl_gpu_create_part(const wasl_gpu_config *config, int64_t node_count,
                         const int64_t *node_tags, const double *node_coordinates,
                         int64_t element_count, const int64_t *element_nodes,
                         int64_t boundary_faces, const int32_t *boundary_donors,
                         const double *boundary_basis, wasl_gpu **handle, char *error,
                         size_t error_length) {
  wasl_b200::PartBoundary part;
  part.faces = boundary_faces;
  part.donors = boundary_donors;
  part.basis = boundary_basis;
  return create_handle(config, node_count, node_tags, node_coordinates, element_count,
                       element_nodes, &part, handle, error, error_length);
}

int wasl_mesh_periodic_trace(int64_t node_count, const int64_t *node_tags,
                             const double *node_coordinates, int64_t element_count,
                             const int64_t *element_nodes, int polynomial_order,
                             int64_t *boundary_faces, int32_t *element, int32_t *edge,
                             int32_t *donors, double *basis, char *error, size_t error_length) {
  std::string message;
  int status = WASL_OK;
  try {
    need(boundary_faces != nullptr, "null pointer");
    need(node_count > 0 && element_count > 0, "mesh: empty node or element list");
    need(node_tags && node_coordinates && element_nodes, "mesh: null array");
    need(polynomial_order >= 0 && polynomial_order <= 3,
         "periodic trace: polynomial order must be 0..3");
    const wasl_b200::TriTopology mesh = wasl_b200::build_triangle_topology(
        node_count, node_tags, node_coordinates, element_count, element_nodes);
    std::int64_t faces = 0;
    for (std::int64_t f = 0; f < mesh.face_count(); ++f)
      faces += mesh.face_right[f] < 0;
    if (!element) { // size query
      *boundary_faces = faces;
    } else {
      need(*boundary_faces == faces, "periodic trace: boundary face count mismatch");
      need(edge && donors && basis, "null pointer");
      const wasl_b200::PeriodicTrace trace = wasl_b200::periodic_trace(mesh, polynomial_order);
      for (std::int64_t f = 0, b = 0; f < mesh.face_count(); ++f)
        if (mesh.face_right[f] < 0) {
          element[b] = mesh.face_left[f];
          edge[b] = mesh.face_left_edge[f];
          ++b;
        }
      std::copy(trace.donors.begin(), trace.donors.end(), donors);
      std::copy(trace.basis.begin(), trace.basis.end(), basis);
    }
  } catch (const wasl_b200::SolverError &e) {
    message = e.what(), status = e.status;
  } catch (const std::invalid_argument &e) {
    message = e.what(), status = WASL_ERR_ARGUMENT;
  } catch (const std::exception &e) {
    message = e.what(), status = WASL_ERR_RUNTIME;
  }
  if (status != WASL_OK)
    copy_message(message, error, error_length);
  return status;
}

void wasl_gpu_destroy(wasl_gpu *h) { delete h; }

const char *wasl_gpu_last_error(const wasl_gpu *h) { return h ? h->error.c_str() : "null handle"; }

int wasl_gpu_sizes(const wasl_gpu *h, int64_t *elements, int64_t *faces, int *modes,
                   int *variables) {
  if (!h)
    return WASL_ERR_ARGUMENT;
  if (elements)
    *elements = h->solver->elements();
  if (faces)
    *faces = h->solver->faces();
  if (modes)
    *modes = h->solver->modes();
  if (variables)
    *variables = h->solver->variables();
  return WASL_OK;
}

int wasl_gpu_element_vertices(const wasl_gpu *h, double *vertices, int64_t count) {
  return guarded(const_cast<wasl_gpu *>(h), [&] {
    need(vertices != nullptr, "null vertex array");
    h->solver->vertices(vertices);
    (void)count;
  });
}

static int64_t state_count(const wasl_gpu *h) {
  return h->solver->elements() * h->solver->modes() * h->solver->variables();
}

int wasl_gpu_set_state(wasl_gpu *h, const double *c, int64_t count) {
  return guarded(h, [&] {
    const wasl_b200::NvtxRange range("wasl_gpu_set_state");
    need(c && count == state_count(h), "state: coefficient count does not match the layout");
    h->solver->set_state(c);
  });
}

int wasl_gpu_get_state(wasl_gpu *h, double *c, int64_t count) {
  return guarded(h, [&] {
    const wasl_b200::NvtxRange range("wasl_gpu_get_state");
    need(c && count == state_count(h), "state: coefficient count does not match the layout");
    h->solver->get_state(c);
  });
}

int wasl_gpu_rule_points(const wasl_gpu *h, int rule_order, int *points) {
  return guarded(const_cast<wasl_gpu *>(h), [&] {
    need(points && rule_order >= 0 && rule_order <= 6, "quadrature: rule order must be 0..6");
    *points = h->solver->rule_points(rule_order);
  });
}

int wasl_gpu_quadrature(const wasl_gpu *h, int rule_order, double *x, double *y, double *w) {
  return guarded(const_cast<wasl_gpu *>(h), [&] {
    need(x && rule_order >= 0 && rule_order <= 6, "quadrature: rule order must be 0..6");
    h->solver->quadrature(rule_order, x, y, w);
  });
}

int wasl_gpu_project(wasl_gpu *h, int rule_order, const double *values, int64_t count) {
  return guarded(h, [&] {
    need(values && rule_order >= 0 && rule_order <= 6, "projection: rule order must be 0..6");
    need(count == h->solver->elements() * h->solver->rule_points(rule_order) *
                      h->solver->variables(),
         "projection: value count must be elements x points x variables");
    h->solver->project(rule_order, values);
  });
}

int wasl_gpu_evaluate(wasl_gpu *h, int rule_order, double *values, int64_t count) {
  return guarded(h, [&] {
    need(values && rule_order >= 0 && rule_order <= 6, "evaluation: rule order must be 0..6");
    need(count == h->solver->elements() * h->solver->rule_points(rule_order) *
                      h->solver->variables(),
         "evaluation: value count must be elements x points x variables");
    h->solver->evaluate(rule_order, values);
  });
}

int wasl_gpu_stable_dt(wasl_gpu *h, double cfl, double *dt) {
  return guarded(h, [&] {
    const wasl_b200::NvtxRange range("wasl_gpu_stable_dt");
    need(dt != nullptr, "null dt");
    *dt = h->solver->stable_dt(cfl);
  });
}

int wasl_gpu_cfl_parts(wasl_gpu *h, double *speed, double *length) {
  return guarded(h, [&] {
    need(speed != nullptr && length != nullptr, "null output");
    h->solver->cfl_parts(*speed, *length);
  });
}

int wasl_gpu_step(wasl_gpu *h, double dt) {
  return guarded(h, [&] {
    const wasl_b200::NvtxRange range("wasl_gpu_step");
    need(std::isfinite(dt), "step: time step is not finite");
    h->solver->step(dt);
  });
}

int wasl_gpu_limit(wasl_gpu *h) {
  return guarded(h, [&] {
    const wasl_b200::NvtxRange range("wasl_gpu_limit");
    h->solver->limit();
  });
}

int wasl_gpu_get_flags(wasl_gpu *h, uint8_t *flags, int64_t count) {
  return guarded(h, [&] {
    need(flags && count == 3 * h->solver->elements(), "flags: count must be 3 x elements");
    h->solver->flags(flags);
  });
}

int wasl_gpu_mass_energy(wasl_gpu *h, double *mass, double *energy) {
  return guarded(h, [&] {
    double m = 0.0, e = 0.0;
    h->solver->mass_energy(m, e);
    if (mass)
      *mass = m;
    if (energy)
      *energy = e;
  });
}

int wasl_gpu_run(wasl_gpu *h, double cfl, double start_time, double end_time, uint64_t max_steps,
                 uint64_t *steps, double *time) {
  return guarded(h, [&] {
    const wasl_b200::NvtxRange range("wasl_gpu_run");
    double t = start_time;
    uint64_t n = 0;
    while (t < end_time && n < max_steps) {
      const double stable = h->solver->stable_dt(cfl);
      const double remaining = end_time - t;
      const double dt = std::min(stable > 0.0 ? stable : remaining, remaining);
      if (dt <= 0.0 || t + dt == t)
        throw std::runtime_error("simulation: timestep cannot advance time");
      h->solver->step(dt);
      t += dt;
      ++n;
    }
    if (steps)
      *steps = n;
    if (time)
      *time = t;
  });
}

int wasl_gpu_run_resident(wasl_gpu *h, double cfl, double start_time, double end_time,
                          uint64_t max_steps, uint64_t *steps, double *time) {
  return guarded(h, [&] {
    const wasl_b200::NvtxRange range("wasl_gpu_run_resident");
    std::uint64_t n = 0;
    double t = start_time;
    h->solver->run_resident(cfl, start_time, end_time, max_steps, n, t);
    if (steps)
      *steps = n;
    if (time)
      *time = t;
  });
}

int wasl_gpu_advance(wasl_gpu *h, double cfl, int64_t steps) {
  return guarded(h, [&] {
    const wasl_b200::NvtxRange range("wasl_gpu_advance");
    need(steps >= 0, "advance: negative step count");
    h->solver->advance(cfl, steps);
  });
}

int wasl_gpu_sync(wasl_gpu *h) {
  return guarded(h, [&] { h->solver->sync(); });
}

int wasl_gpu_state_device(wasl_gpu *h, double **p) {
  return guarded(h, [&] {
    need(p != nullptr, "null pointer");
    *p = h->solver->state_device();
  });
}

int wasl_gpu_element_order(const wasl_gpu *h, int64_t *order, int64_t count) {
  return guarded(const_cast<wasl_gpu *>(h), [&] {
    need(order != nullptr, "null pointer");
    need(count == h->solver->elements(), "element order: count must be the element count");
    h->solver->element_order(order);
  });
}

int wasl_gpu_setup_times(const wasl_gpu *h, double *ms, int count) {
  return guarded(const_cast<wasl_gpu *>(h), [&] {
    need(ms != nullptr, "null pointer");
    need(count >= 0 && count <= WASL_SETUP_PHASES, "setup times: count must be 0..6");
    for (int k = 0; k < count; ++k)
      ms[k] = h->solver->setup_times().ms[k];
  });
}

int wasl_gpu_stencil_transforms(wasl_gpu *h, double *transforms, int64_t count) {
  return guarded(h, [&] {
    need(transforms != nullptr, "null pointer");
    h->solver->stencil_transforms(transforms, count);
  });
}

int wasl_gpu_periodic_trace(wasl_gpu *h, int32_t *donors, double *basis, int64_t points) {
  return guarded(h, [&] {
    need(donors != nullptr && basis != nullptr, "null pointer");
    h->solver->periodic_trace(donors, basis, points);
  });
}

int wasl_gpu_stream(wasl_gpu *h, void **s) {
  return guarded(h, [&] {
    need(s != nullptr, "null pointer");
    *s = reinterpret_cast<void *>(h->solver->stream());
  });
}

int wasl_gpu_tuning(const wasl_gpu *h, int *choice, double *ms, int capacity, int *count) {
  return guarded(const_cast<wasl_gpu *>(h), [&] {
    need(choice && count && (ms || capacity <= 0), "tuning: null output");
    int n = 0;
    *choice = h->solver->kernel_choice(ms, capacity, n);
    *count = n;
  });
}

int wasl_gpu_indicator_features(const wasl_gpu *h, int *features) {
  return guarded(const_cast<wasl_gpu *>(h), [&] {
    need(features != nullptr, "indicator features: null output");
    *features = h->solver->indicator_features();
  });
}

int wasl_gpu_indicator_data(wasl_gpu *h, float *features, uint8_t *labels, int64_t count) {
  return guarded(h, [&] {
    need(features && labels && count == h->solver->elements(),
         "indicator data: count must be the number of elements");
    h->solver->indicator_data(features, labels);
  });
}

int wasl_gpu_indicator_kernel(wasl_gpu *h, int kernel) {
  return guarded(h, [&] { h->solver->set_indicator_kernel(kernel); });
}

int wasl_gpu_set_indicator(wasl_gpu *h, const float *weights, int64_t count, double lo,
                           double hi) {
  return guarded(h, [&] {
    need(weights != nullptr, "set indicator: null weights");
    h->solver->set_indicator(weights, count, lo, hi);
  });
}

int wasl_gpu_indicator_logits(wasl_gpu *h, float *logits, int64_t count) {
  return guarded(h, [&] {
    need(logits && count == h->solver->elements(),
         "indicator logits: count must be the number of elements");
    h->solver->indicator_logits(logits);
  });
}

int wasl_gpu_indicator_stats(wasl_gpu *h, uint64_t *stats, int reset) {
  return guarded(h, [&] {
    need(stats != nullptr, "indicator stats: null output");
    unsigned long long s[6];
    h->solver->indicator_stats(s, reset != 0);
    for (int i = 0; i < 6; ++i)
      stats[i] = s[i];
  });
}

int wasl_gpu_profile_begin(wasl_gpu *h) {
  return guarded(h, [&] { h->solver->profile_begin(); });
}

int wasl_gpu_profile_stages(const wasl_gpu *h, double *stage_ms) {
  return guarded(const_cast<wasl_gpu *>(h), [&] {
    need(stage_ms != nullptr, "profile stages: null output");
    for (int k = 0; k < 3; ++k)
      stage_ms[k] = h->solver->profile_stage_ms()[k];
  });
}

int wasl_gpu_profile_end(wasl_gpu *h, double *stage_ms, int64_t *stage_kernels,
                         int64_t *launches) {
  return guarded(h, [&] {
    double ms = 0.0;
    std::int64_t k = 0, n = 0;
    h->solver->profile_end(ms, k, n);
    if (stage_ms)
      *stage_ms = ms;
    if (stage_kernels)
      *stage_kernels = k;
    if (launches)
      *launches = n;
  });
}

int wasl_gpu_write_checkpoint(wasl_gpu *h, const char *path, double time, uint64_t step,
                              const char *prepared_mesh) {
  return guarded(h, [&] {
    need(path != nullptr, "checkpoint: null path");
    std::vector<double> c(state_count(h));
    h->solver->get_state(c.data());
    std::ofstream o(path, std::ios::binary | std::ios::trunc);
    if (!o)
      throw std::runtime_error(std::string("checkpoint write: cannot open ") + path);
    const std::string mesh = prepared_mesh ? prepared_mesh : "";
    o.write(kMagic, sizeof(kMagic));
    put<int32_t>(o, 2);
    put<double>(o, time);
    put<uint64_t>(o, step);
    put<uint64_t>(o, h->solver->variables());
    put<uint64_t>(o, h->solver->modes());
    put<uint64_t>(o, h->solver->elements());
    put<uint64_t>(o, mesh.size());
    o.write(mesh.data(), static_cast<std::streamsize>(mesh.size()));
    put<uint64_t>(o, c.size());
    o.write(reinterpret_cast<const char *>(c.data()),
            static_cast<std::streamsize>(c.size() * sizeof(double)));
    put<int32_t>(o, 0);                          // partition_rank
    put<int32_t>(o, 1);                          // partition_rank_count
    put<uint64_t>(o, h->solver->elements());     // global_element_count
    put<uint64_t>(o, 0);                         // element_indices: identity
    if (!o)
      throw std::runtime_error(std::string("checkpoint write: failed ") + path);
  });
}

int wasl_gpu_read_checkpoint(wasl_gpu *h, const char *path, double *time, uint64_t *step) {
  return guarded(h, [&] {
    need(path != nullptr, "checkpoint: null path");
    std::ifstream i(path, std::ios::binary);
    if (!i)
      throw std::runtime_error(std::string("checkpoint read: file does not exist: ") + path);
    char magic[8];
    i.read(magic, 8);
    if (!i || std::memcmp(magic, kMagic, 8) != 0)
      throw std::runtime_error("checkpoint read: not a checkpoint file");
    const int32_t version = get<int32_t>(i);
    if (version != 2)
      throw std::runtime_error("checkpoint read: unsupported format_version");
    const double t = get<double>(i);
    const uint64_t s = get<uint64_t>(i);
    const uint64_t nv = get<uint64_t>(i), nm = get<uint64_t>(i), ne = get<uint64_t>(i);
    const uint64_t mesh_len = get<uint64_t>(i);
    std::string mesh(mesh_len, '\0');
    i.read(mesh.data(), static_cast<std::streamsize>(mesh_len));
    const uint64_t n = get<uint64_t>(i);
    if (nv != static_cast<uint64_t>(h->solver->variables()) ||
        nm != static_cast<uint64_t>(h->solver->modes()) ||
        ne != static_cast<uint64_t>(h->solver->elements()) || n != nv * nm * ne)
      throw std::runtime_error(
          "simulation restart: checkpoint layout or mesh provenance mismatch");
    std::vector<double> c(n);
    i.read(reinterpret_cast<char *>(c.data()), static_cast<std::streamsize>(n * sizeof(double)));
    if (!i)
      throw std::runtime_error("checkpoint read: truncated file");
    h->solver->set_state(c.data());
    if (time)
      *time = t;
    if (step)
      *step = s;
  });
}

} // extern "C"
