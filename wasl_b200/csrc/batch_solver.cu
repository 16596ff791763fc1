// Batched 2D Euler: many independent triangle meshes of uneven size advanced
// together in the mixed form.
//
// Cases are grouped by polynomial order; each group's meshes are laid end to
// end as one disconnected mesh (elements of a case contiguous, neighbour and
// periodic indices offset), so every kernel of the single-case path runs on a
// group unchanged.  Each case is cut into tiles that never straddle two cases:
// the tile list is the work list of the fused tile kernel (one CTA per tile,
// equal cost per tile whatever the case sizes), and each tile carries its case,
// whose own CFL time step the kernel applies.  A step is
//   per group: the per-case CFL speed over the group's tiles;
//   dt per case (and elapsed time);
//   three stages: per group the tile kernel (and the stage limiter);
// enqueued once and captured in a CUDA graph that each later step replays.
// The tile shape is autotuned per group (polynomial order) before capture.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

#include "autotune.hpp"
#include "batch.hpp"
#include "kernels.hpp"
#include "tri_setup.hpp"
#include "tri_tables.hpp"

namespace wasl_b200 {

BatchSolver::Group::Group() = default;
BatchSolver::Group::~Group() = default;

namespace {

// Everything one case contributes, built on the host.
struct CaseSetup {
  TriTopology mesh;
  TriSlots slots;
  TileSlotArrays tile;
  std::vector<float> basis32;
  LimiterStencil stencil;
  double length = 0.0;
  std::string error;
};

template <typename T> void append(std::vector<T> &dst, const std::vector<T> &src) {
  dst.insert(dst.end(), src.begin(), src.end());
}

// Rows [rows][n] of a per-case array placed at column `offset` of [rows][total].
template <typename T>
void place_rows(std::vector<T> &dst, const std::vector<T> &src, int rows, std::int64_t n,
                std::int64_t offset, std::int64_t total) {
  for (int r = 0; r < rows; ++r)
    std::copy(src.begin() + r * n, src.begin() + (r + 1) * n, dst.begin() + r * total + offset);
}

} // namespace

BatchSolver::BatchSolver(const wasl_batch_config &cfg, std::int64_t case_count, const int *orders,
                         const std::int64_t *node_counts, const std::int64_t *node_tags,
                         const double *node_xy, const std::int64_t *element_counts,
                         const std::int64_t *element_nodes)
    : cfg_(cfg), cases_(case_count) {
  if (case_count <= 0)
    throw SolverError(WASL_ERR_ARGUMENT, "batch: no cases");
  if (cfg.boundary != WASL_PERIODIC && cfg.boundary != WASL_TRANSMISSIVE)
    throw SolverError(WASL_ERR_ARGUMENT, "batch: boundaries must be periodic or transmissive");
  if (cfg.tile_shape < 0 || cfg.tile_shape > euler_tri_tile_shapes())
    throw SolverError(WASL_ERR_ARGUMENT, "batch: unknown tile shape");
  if (cfg.tile_shape > 0 && euler_tri_tile_is_patch(cfg.tile_shape - 1))
    throw SolverError(WASL_ERR_ARGUMENT, "batch: the patch kernel's shapes are for single cases");
  for (std::int64_t c = 0; c < case_count; ++c)
    if (!euler_tri_mixed_supported(orders[c], 0))
      throw SolverError(WASL_ERR_ARGUMENT, "batch: polynomial order must be 1..3 (case " +
                                               std::to_string(c) + ")");
  cuda_check(cudaSetDevice(cfg.device), "cudaSetDevice");
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");

  // Host setup, cases in parallel.
  std::vector<std::int64_t> node_begin(case_count + 1, 0), elem_begin(case_count + 1, 0);
  for (std::int64_t c = 0; c < case_count; ++c) {
    node_begin[c + 1] = node_begin[c] + node_counts[c];
    elem_begin[c + 1] = elem_begin[c] + element_counts[c];
  }
  std::vector<CaseSetup> setup(case_count);
  {
    const unsigned workers = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(),
                                                             static_cast<unsigned>(case_count)));
    std::vector<std::thread> pool;
    std::atomic<std::int64_t> next{0};
    for (unsigned w = 0; w < workers; ++w)
      pool.emplace_back([&] {
        for (std::int64_t c = next++; c < case_count; c = next++) {
          CaseSetup &cs = setup[c];
          try {
            const int p = orders[c], QF = p + 1, M = tri_modes(p);
            cs.mesh = build_triangle_topology(node_counts[c], node_tags + node_begin[c],
                                              node_xy + 2 * node_begin[c], element_counts[c],
                                              element_nodes + 3 * elem_begin[c]);
            bool has_boundary = false;
            for (std::int64_t f = 0; f < cs.mesh.face_count(); ++f)
              has_boundary |= cs.mesh.face_right[f] < 0;
            PeriodicTrace trace;
            const bool periodic = has_boundary && cfg.boundary == WASL_PERIODIC;
            if (periodic)
              trace = periodic_trace(cs.mesh, p);
            cs.slots = build_tri_slots(cs.mesh, periodic ? &trace : nullptr, QF, M);
            if (periodic && !pair_periodic_faces(cs.mesh, QF, cs.slots, cs.basis32))
              throw SolverError(WASL_ERR_ARGUMENT, "batch: periodic faces do not pair one to one");
            cs.tile = build_tile_slots(cs.mesh, cs.slots, cfg.boundary, QF);
            if (cfg.limiting)
              cs.stencil = triangle_stencil(cs.mesh, p, trace.donors);
            cs.length = minimum_altitude(cs.mesh);
          } catch (const std::exception &e) {
            cs.error = "case " + std::to_string(c) + ": " + e.what();
          }
        }
      });
    for (auto &t : pool)
      t.join();
  }
  for (const auto &cs : setup)
    if (!cs.error.empty())
      throw SolverError(WASL_ERR_ARGUMENT, "batch: " + cs.error);

  // Groups by polynomial order, concatenated.
  case_group_.assign(case_count, -1);
  case_offset_.assign(case_count, 0);
  std::vector<double> lengths(case_count);
  std::vector<int> case_p(case_count);
  for (int p = 1; p <= 3; ++p) {
    std::vector<std::int64_t> members;
    for (std::int64_t c = 0; c < case_count; ++c)
      if (orders[c] == p)
        members.push_back(c);
    if (members.empty())
      continue;
    auto g = std::make_unique<Group>();
    g->p = p;
    g->M = tri_modes(p);
    g->rule = cfg.reduced_volume_rule ? p : p + 2;
    const int QF = p + 1, M = g->M;
    std::int64_t ne = 0, nb = 0;
    for (std::int64_t c : members) {
      case_group_[c] = static_cast<int>(groups_.size());
      case_offset_[c] = ne;
      ne += setup[c].mesh.element_count;
    }
    g->ne = ne;
    g->cases = members;
    std::vector<double> geo(5 * ne), slot_geo(9 * ne);
    std::vector<std::int32_t> nbr(3 * ne), aux(3 * ne), neighbors;
    std::vector<std::uint8_t> code(3 * ne);
    std::vector<float> basis32;
    std::vector<double> basis64, transforms, nx, ny;
    for (std::int64_t c : members) {
      const CaseSetup &cs = setup[c];
      const std::int64_t n = cs.mesh.element_count, off = case_offset_[c];
      place_rows(geo, cs.slots.geo, 5, n, off, ne);
      place_rows(slot_geo, cs.slots.slot_geo, 9, n, off, ne);
      std::vector<std::int32_t> cn = cs.tile.nbr, ca = cs.tile.aux;
      for (auto &v : cn)
        if (v >= 0)
          v += static_cast<std::int32_t>(off);
      for (auto &v : ca)
        v += static_cast<std::int32_t>(nb);
      place_rows(nbr, cn, 3, n, off, ne);
      place_rows(aux, ca, 3, n, off, ne);
      place_rows(code, cs.tile.code, 3, n, off, ne);
      append(basis32, cs.basis32);
      if (!cs.basis32.empty())
        append(basis64, cs.slots.donor_basis);
      nb += static_cast<std::int64_t>(cs.basis32.size()) / (QF * M);
      if (cfg.limiting) {
        std::vector<std::int32_t> sn = cs.stencil.neighbors;
        for (auto &v : sn)
          if (v >= 0)
            v += static_cast<std::int32_t>(off);
        append(neighbors, sn);
        append(transforms, cs.stencil.transforms);
        append(nx, cs.stencil.normal_x);
        append(ny, cs.stencil.normal_y);
      }
      lengths[c] = cs.length;
      case_p[c] = p;
    }
    std::vector<std::int32_t> element_case(ne);
    for (std::int64_t c : members)
      std::fill(element_case.begin() + case_offset_[c],
                element_case.begin() + case_offset_[c] + setup[c].mesh.element_count,
                static_cast<std::int32_t>(c));
    g->element_case.upload(element_case, stream_);
    g->geo.upload(geo, stream_);
    g->slot_geo.upload(slot_geo, stream_);
    g->tile_nbr.upload(nbr, stream_);
    g->tile_aux.upload(aux, stream_);
    g->tile_code.upload(code, stream_);
    if (!basis32.empty()) {
      g->basis32.upload(basis32, stream_);
      g->basis64.upload(basis64, stream_);
    }
    std::vector<unsigned char> table(euler_tri_face_table_bytes(p, true));
    fill_euler_tri_face_table(p, true, table.data());
    g->face_table.upload(table, stream_);
    std::vector<unsigned char> table64(euler_tri_face_table_bytes(p, false));
    fill_euler_tri_face_table(p, false, table64.data());
    g->face_table64.upload(table64, stream_);
    upload_euler_tri_tables_mixed(p, g->rule);
    prepare_euler_tri_stage_tile(p, g->rule);
    if (cfg.limiting) {
      const LimiterStencil &first = setup[members[0]].stencil;
      g->highest_degree_begin = first.highest_degree_begin;
      g->check_points = first.check_point_count();
      g->neighbors.upload(neighbors, stream_);
      g->transforms.upload(transforms, stream_);
      g->normal_x.upload(nx, stream_);
      g->normal_y.upload(ny, stream_);
      g->check.upload(first.check_basis, stream_);
      g->check_bound.upload(positivity_check_bound(first.check_basis, M), stream_);
      g->limited.resize(static_cast<std::size_t>(ne) * 4 * M);
      g->troubled.resize(ne);
      g->count.resize(1);
      g->flags.resize(ne);
    }
    for (auto *b : {&g->u, &g->e, &g->s})
      b->resize(static_cast<std::size_t>(4) * M * ne);
    if (cfg.limiting)
      g->rough.resize(ne + 1); // rough list, then its count
    cuda_check(cudaMemsetAsync(g->u.get(), 0, g->u.size() * sizeof(double), stream_), "memset");
    // Work lists, one per tile size of the launch shapes.
    for (int shape = 0; shape < euler_tri_tile_shapes(); ++shape) {
      const int T = euler_tri_tile_elements(shape);
      std::vector<TileWork> work;
      for (std::int64_t c : members) {
        const std::int64_t n = setup[c].mesh.element_count, off = case_offset_[c];
        for (std::int64_t s = 0; s < n; s += T) {
          TileWork w;
          w.first = static_cast<std::int32_t>(off + s);
          w.count = static_cast<std::int32_t>(std::min<std::int64_t>(T, n - s));
          w.case_id = static_cast<std::int32_t>(c);
          work.push_back(w);
        }
      }
      g->work_count[shape] = static_cast<std::int64_t>(work.size());
      g->work[shape].upload(work, stream_);
    }
    total_elements_ += ne;
    total_dof_ += 4LL * M * ne;
    groups_.push_back(std::move(g));
  }
  // Per-case meshes are kept for quadrature and projection only.
  meshes_.resize(case_count);
  for (std::int64_t c = 0; c < case_count; ++c) {
    meshes_[c].element_count = setup[c].mesh.element_count;
    meshes_[c].maps = std::move(setup[c].mesh.maps);
  }
  d_length_.upload(lengths, stream_);
  d_p_.upload(case_p, stream_);
  d_dt_.resize(case_count);
  d_time_.resize(case_count);
  d_speed_.resize(case_count);
  d_error_.resize(1);
  d_status_.resize(case_count);
  cuda_check(cudaMemsetAsync(d_status_.get(), 0, case_count * sizeof(int), stream_), "memset");
  cuda_check(cudaMemsetAsync(d_dt_.get(), 0, case_count * sizeof(double), stream_), "memset");
  cuda_check(cudaMemsetAsync(d_time_.get(), 0, case_count * sizeof(double), stream_), "memset");
  cuda_check(cudaMemsetAsync(d_speed_.get(), 0, case_count * sizeof(unsigned long long), stream_),
             "memset");
  cuda_check(cudaMemsetAsync(d_error_.get(), 0, sizeof(unsigned long long), stream_), "memset");
  cuda_check(cudaStreamSynchronize(stream_), "batch setup");
}

BatchSolver::~BatchSolver() {
  if (graph_exec_)
    cudaGraphExecDestroy(graph_exec_);
  if (stream_)
    cudaStreamDestroy(stream_);
}

std::int64_t BatchSolver::case_elements(std::int64_t c) const { return meshes_.at(c).element_count; }

int BatchSolver::case_modes(std::int64_t c) const { return groups_.at(case_group_.at(c))->M; }

void BatchSolver::check_case(std::int64_t c) const {
  if (c < 0 || c >= cases_)
    throw SolverError(WASL_ERR_ARGUMENT, "batch: case index out of range");
}

void BatchSolver::copy_case(std::int64_t c, double *host, bool to_device) {
  check_case(c);
  const Group &g = *groups_[case_group_[c]];
  const std::int64_t n = meshes_[c].element_count;
  double *dev = g.u.get() + case_offset_[c];
  const std::size_t width = n * sizeof(double), pitch_dev = g.ne * sizeof(double);
  if (to_device)
    cuda_check(cudaMemcpy2DAsync(dev, pitch_dev, host, width, width, 4 * g.M,
                                 cudaMemcpyHostToDevice, stream_),
               "batch set_state");
  else
    cuda_check(cudaMemcpy2DAsync(host, width, dev, pitch_dev, width, 4 * g.M,
                                 cudaMemcpyDeviceToHost, stream_),
               "batch get_state");
  cuda_check(cudaStreamSynchronize(stream_), "batch state copy");
}

void BatchSolver::set_state(std::int64_t c, const double *host) {
  copy_case(c, const_cast<double *>(host), true);
}

void BatchSolver::get_state(std::int64_t c, double *host) { copy_case(c, host, false); }

void BatchSolver::quadrature(std::int64_t c, int rule, double *x, double *y, double *w) const {
  check_case(c);
  tri_quadrature(meshes_[c], rule, x, y, w);
}

void BatchSolver::project(std::int64_t c, int rule, const double *values) {
  check_case(c);
  const Group &g = *groups_[case_group_[c]];
  const std::vector<double> coeffs = tri_project(meshes_[c], g.p, 4, rule, values);
  set_state(c, coeffs.data());
}

StageArgs BatchSolver::stage_args(const Group &g, int stage) const {
  StageArgs a;
  a.mesh.ne = g.ne;
  a.mesh.geo = g.geo.get();
  a.mesh.slot_geo = g.slot_geo.get();
  a.mesh.boundary = cfg_.boundary;
  a.boundary.basis32 = g.basis32.get();
  a.mesh.donor_basis = g.basis64.get();
  a.face_table = g.face_table.get();
  a.face_table64 = g.face_table64.get();
  a.tile.nbr = g.tile_nbr.get();
  a.tile.code = g.tile_code.get();
  a.tile.aux = g.tile_aux.get();
  // FP64 face islands at discontinuities (the rough pass), with the limiter.
  a.rough = cfg_.limiting ? g.rough.get() : nullptr;
  a.rough_count = a.rough ? g.rough.get() + g.ne : nullptr;
  a.element_case = g.element_case.get();
  a.work = g.work[g.shape].get();
  a.work_count = g.work_count[g.shape];
  a.case_dt = d_dt_.get();
  a.gamma = cfg_.heat_capacity_ratio;
  a.stage = stage;
  const double *ins[3] = {g.u.get(), g.e.get(), g.s.get()};
  double *outs[3] = {g.e.get(), g.s.get(), g.u.get()};
  a.in = ins[stage];
  a.out = outs[stage];
  a.u0 = g.u.get();
  a.sense = cfg_.limiting ? 1 : 0;
  a.threshold = cfg_.sensor_threshold;
  a.highest_degree_begin = g.highest_degree_begin;
  a.flags = g.flags.get();
  a.troubled = g.troubled.get();
  a.troubled_count = g.count.get();
  a.error = d_error_.get();
  return a;
}

LimitArgs BatchSolver::limit_args(const Group &g, double *state) const {
  LimitArgs l;
  l.ne = g.ne;
  l.state = state;
  l.troubled = g.troubled.get();
  l.troubled_count = g.count.get();
  l.neighbors = g.neighbors.get();
  l.transforms = g.transforms.get();
  l.normal_x = g.normal_x.get();
  l.normal_y = g.normal_y.get();
  l.check_basis = g.check.get();
  l.check_points = g.check_points;
  l.gamma = cfg_.heat_capacity_ratio;
  l.density_floor = cfg_.density_floor;
  l.pressure_floor = cfg_.pressure_floor;
  l.limited = g.limited.get();
  l.error = d_error_.get();
  l.positivity_all = cfg_.positivity_all ? 1 : 0;
  l.flags = g.flags.get();
  l.relative_floor = kMixedRelativeFloor;
  l.case_status = d_status_.get();
  l.check_bound = g.check_bound.get();
  l.element_case = g.element_case.get();
  return l;
}

void BatchSolver::tune() {
  for (auto &gp : groups_) {
    Group &g = *gp;
    if (cfg_.tile_shape > 0) {
      g.shape = cfg_.tile_shape - 1;
      continue;
    }
    // Each shape runs the first stage of the current state into scratch
    // (u^n read, not written; no sensing, dt 0).
    cuda_check(cudaMemsetAsync(d_dt_.get(), 0, cases_ * sizeof(double), stream_), "memset");
    const std::string key = "batch_tile/p" + std::to_string(g.p) + "/rule" +
                            std::to_string(g.rule) + "/bnd" + std::to_string(cfg_.boundary) +
                            "/size" + std::to_string(size_class(g.ne));
    std::vector<int> shapes; // the tile kernels' shapes (not the patch kernel's)
    for (int shape = 0; shape < euler_tri_tile_shapes(); ++shape)
      if (!euler_tri_tile_is_patch(shape))
        shapes.push_back(shape);
    const TuneResult timed = autotune(key, static_cast<int>(shapes.size()), [&](int i) {
      g.shape = shapes[i];
      StageArgs a = stage_args(g, 0);
      a.sense = 0;
      launch_euler_tri_stage_tile(g.p, g.rule, shapes[i], a, stream_);
    }, stream_);
    // By shape (0 for the shapes not timed).
    g.tuning.ms.assign(euler_tri_tile_shapes(), 0.0);
    for (std::size_t i = 0; i < shapes.size(); ++i)
      g.tuning.ms[shapes[i]] = timed.ms[i];
    g.shape = g.tuning.choice = shapes[timed.choice];
  }
}

void BatchSolver::enqueue_step(double cfl) {
  for (auto &gp : groups_) {
    const Group &g = *gp;
    launch_batch_speed(g.u.get(), g.ne, g.M, cfg_.heat_capacity_ratio, g.work[g.shape].get(),
                       g.work_count[g.shape], d_speed_.get(), d_error_.get(), d_status_.get(),
                       stream_);
  }
  launch_dt_from_speed(cases_, d_speed_.get(), cfl, d_length_.get(), d_p_.get(), 0.0, 0,
                       d_dt_.get(), d_time_.get(), d_status_.get(), stream_);
  launches_per_step_ = static_cast<std::int64_t>(groups_.size()) + 1;
  for (int k = 0; k < 3; ++k)
    for (auto &gp : groups_) {
      Group &g = *gp;
      if (cfg_.limiting)
        cuda_check(cudaMemsetAsync(g.count.get(), 0, sizeof(std::int32_t), stream_), "count");
      const StageArgs a = stage_args(g, k);
      launch_euler_tri_stage_tile(g.p, g.rule, g.shape, a, stream_);
      launches_per_step_ += a.rough ? 2 : 1;
      if (cfg_.limiting) {
        launch_limit_f64(g.M, 3, limit_args(g, a.out), stream_);
        launches_per_step_ += cfg_.positivity_all ? 3 : 2;
      }
    }
}

void BatchSolver::advance(double cfl, std::int64_t steps) {
  if (steps <= 0)
    return;
  if (!tuned_) {
    tune();
    tuned_ = true;
  }
  std::int64_t done = 0;
  if (cfg_.use_graph) {
    if (!graph_exec_ || graph_cfl_ != cfl) {
      if (graph_exec_) {
        cuda_check(cudaGraphExecDestroy(graph_exec_), "graph destroy");
        graph_exec_ = nullptr;
      }
      cudaGraph_t graph = nullptr;
      cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
      {
        // Ends the capture (and drops the partial graph) if enqueuing throws,
        // so the stream leaves capture mode and later calls still work.
        struct CaptureGuard {
          cudaStream_t stream;
          bool open = true;
          ~CaptureGuard() {
            if (!open)
              return;
            cudaGraph_t partial = nullptr;
            if (cudaStreamEndCapture(stream, &partial) == cudaSuccess && partial)
              cudaGraphDestroy(partial);
          }
        } guard{stream_};
        enqueue_step(cfl);
        guard.open = false;
      }
      cuda_check(cudaStreamEndCapture(stream_, &graph), "capture end");
      cuda_check(cudaGraphInstantiate(&graph_exec_, graph, 0), "graph instantiate");
      cuda_check(cudaGraphDestroy(graph), "graph destroy");
      graph_cfl_ = cfl;
    }
    for (; done < steps; ++done)
      cuda_check(cudaGraphLaunch(graph_exec_, stream_), "graph launch");
  } else {
    for (; done < steps; ++done)
      enqueue_step(cfl);
  }
  launches_ += launches_per_step_ * steps;
  check_error();
}

void BatchSolver::limit() {
  if (!cfg_.limiting)
    return;
  for (auto &gp : groups_) {
    Group &g = *gp;
    if (g.p == 0)
      continue;
    cuda_check(cudaMemsetAsync(g.count.get(), 0, sizeof(std::int32_t), stream_), "count");
    SenseArgs sa;
    sa.ne = g.ne;
    sa.state = g.u.get();
    sa.threshold = cfg_.sensor_threshold;
    sa.highest_degree_begin = g.highest_degree_begin;
    sa.flags = g.flags.get();
    sa.troubled = g.troubled.get();
    sa.troubled_count = g.count.get();
    launch_sense_f64(g.M, sa, stream_);
    launch_limit_f64(g.M, 3, limit_args(g, g.u.get()), stream_);
  }
  check_error();
}

void BatchSolver::check_error() {
  unsigned long long word = 0;
  cuda_check(cudaMemcpyAsync(&word, d_error_.get(), sizeof(word), cudaMemcpyDeviceToHost, stream_),
             "error word");
  cuda_check(cudaStreamSynchronize(stream_), "batch step");
  if (word) {
    cuda_check(cudaMemsetAsync(d_error_.get(), 0, sizeof(word), stream_), "memset");
    cuda_check(cudaStreamSynchronize(stream_), "batch step");
    // The element index is the group's; name the case it belongs to.
    throw_device_error(word);
  }
}

void BatchSolver::status(int *out) {
  cuda_check(cudaMemcpyAsync(out, d_status_.get(), cases_ * sizeof(int), cudaMemcpyDeviceToHost,
                             stream_),
             "status");
  cuda_check(cudaStreamSynchronize(stream_), "status");
}

void BatchSolver::times(double *time, double *dt) {
  if (time)
    cuda_check(cudaMemcpyAsync(time, d_time_.get(), cases_ * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "times");
  if (dt)
    cuda_check(cudaMemcpyAsync(dt, d_dt_.get(), cases_ * sizeof(double), cudaMemcpyDeviceToHost,
                               stream_),
               "dts");
  cuda_check(cudaStreamSynchronize(stream_), "times");
}

int BatchSolver::tuning(int p, double *ms, int capacity, int &count) const {
  for (const auto &g : groups_)
    if (g->p == p) {
      count = static_cast<int>(g->tuning.ms.size());
      for (int i = 0; i < count && i < capacity; ++i)
        ms[i] = g->tuning.ms[i];
      return g->shape;
    }
  count = 0;
  return -1;
}

} // namespace wasl_b200
