// extern "C" entry points of the batched solver (declared in include/wasl_b200.h).
#include <cstring>
#include <stdexcept>

#include "batch.hpp"

struct wasl_batch {
  std::unique_ptr<wasl_b200::BatchSolver> solver;
  std::string error;
};

namespace {

template <typename F> int guarded(wasl_batch *h, F &&body) {
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

} // namespace

extern "C" {

void wasl_batch_config_default(wasl_batch_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->heat_capacity_ratio = 1.4;
  c->boundary = WASL_TRANSMISSIVE;
  c->sensor_threshold = 1e-3;
  c->density_floor = 1e-10;
  c->pressure_floor = 1e-10;
  c->reduced_volume_rule = 1;
  c->use_graph = 1;
}

int wasl_batch_create(const wasl_batch_config *config, int64_t case_count, const int *orders,
                      const int64_t *node_counts, const int64_t *node_tags,
                      const double *node_coordinates, const int64_t *element_counts,
                      const int64_t *element_nodes, wasl_batch **handle, char *error,
                      size_t error_length) {
  auto fail = [&](int status, const char *message) {
    if (error && error_length) {
      std::strncpy(error, message, error_length - 1);
      error[error_length - 1] = '\0';
    }
    return status;
  };
  if (!config || !orders || !node_counts || !node_tags || !node_coordinates || !element_counts ||
      !element_nodes || !handle)
    return fail(WASL_ERR_ARGUMENT, "batch: null argument");
  *handle = nullptr;
  try {
    auto *h = new wasl_batch;
    try {
      h->solver = std::make_unique<wasl_b200::BatchSolver>(*config, case_count, orders,
                                                           node_counts, node_tags,
                                                           node_coordinates, element_counts,
                                                           element_nodes);
    } catch (...) {
      delete h;
      throw;
    }
    *handle = h;
    return WASL_OK;
  } catch (const wasl_b200::SolverError &e) {
    return fail(e.status, e.what());
  } catch (const std::invalid_argument &e) {
    return fail(WASL_ERR_ARGUMENT, e.what());
  } catch (const std::exception &e) {
    return fail(WASL_ERR_RUNTIME, e.what());
  }
}

void wasl_batch_destroy(wasl_batch *h) { delete h; }

const char *wasl_batch_last_error(const wasl_batch *h) { return h ? h->error.c_str() : "null handle"; }

int wasl_batch_sizes(const wasl_batch *h, int64_t *cases, int64_t *elements, int64_t *dof) {
  return guarded(const_cast<wasl_batch *>(h), [&] {
    if (cases)
      *cases = h->solver->cases();
    if (elements)
      *elements = h->solver->total_elements();
    if (dof)
      *dof = h->solver->total_dof();
  });
}

int wasl_batch_case_size(const wasl_batch *h, int64_t c, int64_t *elements, int *modes) {
  return guarded(const_cast<wasl_batch *>(h), [&] {
    need(c >= 0 && c < h->solver->cases(), "batch: case index out of range");
    if (elements)
      *elements = h->solver->case_elements(c);
    if (modes)
      *modes = h->solver->case_modes(c);
  });
}

int wasl_batch_set_state(wasl_batch *h, int64_t c, const double *coefficients, int64_t count) {
  return guarded(h, [&] {
    need(c >= 0 && c < h->solver->cases(), "batch: case index out of range");
    need(coefficients && count == 4 * h->solver->case_modes(c) * h->solver->case_elements(c),
         "batch set_state: wrong coefficient count");
    h->solver->set_state(c, coefficients);
  });
}

int wasl_batch_get_state(wasl_batch *h, int64_t c, double *coefficients, int64_t count) {
  return guarded(h, [&] {
    need(c >= 0 && c < h->solver->cases(), "batch: case index out of range");
    need(coefficients && count == 4 * h->solver->case_modes(c) * h->solver->case_elements(c),
         "batch get_state: wrong coefficient count");
    h->solver->get_state(c, coefficients);
  });
}

int wasl_batch_quadrature(const wasl_batch *h, int64_t c, int rule_order, double *x, double *y,
                          double *weights) {
  return guarded(const_cast<wasl_batch *>(h), [&] {
    need(x && y, "batch quadrature: null output");
    need(rule_order >= 0 && rule_order <= 6, "batch quadrature: rule order must be 0..6");
    h->solver->quadrature(c, rule_order, x, y, weights);
  });
}

int wasl_batch_project(wasl_batch *h, int64_t c, int rule_order, const double *values,
                       int64_t count) {
  return guarded(h, [&] {
    need(c >= 0 && c < h->solver->cases(), "batch: case index out of range");
    need(rule_order >= 0 && rule_order <= 6, "batch project: rule order must be 0..6");
    need(values && count == 4LL * (rule_order + 1) * (rule_order + 1) * h->solver->case_elements(c),
         "batch project: wrong value count");
    h->solver->project(c, rule_order, values);
  });
}

int wasl_batch_limit(wasl_batch *h) {
  return guarded(h, [&] { h->solver->limit(); });
}

int wasl_batch_advance(wasl_batch *h, double cfl, int64_t steps) {
  return guarded(h, [&] {
    need(cfl > 0.0 && steps >= 0, "batch advance: cfl must be positive and steps non-negative");
    const wasl_b200::NvtxRange range("wasl_batch_advance");
    h->solver->advance(cfl, steps);
  });
}

int wasl_batch_status(wasl_batch *h, int *status, int64_t count) {
  return guarded(h, [&] {
    need(status && count == h->solver->cases(), "batch status: count must be the number of cases");
    h->solver->status(status);
  });
}

int wasl_batch_times(wasl_batch *h, double *time, double *dt, int64_t count) {
  return guarded(h, [&] {
    need(count == h->solver->cases(), "batch times: count must be the number of cases");
    h->solver->times(time, dt);
  });
}

int wasl_batch_tuning(const wasl_batch *h, int p, int *choice, double *ms, int capacity,
                      int *count) {
  return guarded(const_cast<wasl_batch *>(h), [&] {
    need(choice && count && (ms || capacity <= 0), "batch tuning: null output");
    int n = 0;
    *choice = h->solver->tuning(p, ms, capacity, n);
    *count = n;
  });
}

int wasl_batch_launches(const wasl_batch *h, int64_t *per_step, int *graph, int64_t *total) {
  return guarded(const_cast<wasl_batch *>(h), [&] {
    if (per_step)
      *per_step = h->solver->launches_per_step();
    if (graph)
      *graph = h->solver->graph() ? 1 : 0;
    if (total)
      *total = h->solver->launches();
  });
}

int wasl_batch_stream(wasl_batch *h, void **stream) {
  return guarded(h, [&] {
    need(stream != nullptr, "batch stream: null output");
    *stream = h->solver->stream();
  });
}

} // extern "C"
