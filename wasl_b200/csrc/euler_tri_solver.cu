// 2D Euler on triangles: setup data on the device and the SSP-RK3 step.
//
// Mirrors the reference case driver (cpp/src/case/euler_triangle.cpp:16-49):
// periodic trace and limiter stencil built once, then per step the CFL time
// step (cfl_timestep.cpp:78-84) and ssp_rk3_step with the stage limiter
// (ssp_rk3.hpp:37-61, euler_state_operations.cpp:26-34).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>

#include "autotune.hpp"
#include "basis.hpp"
#include "kernels.hpp"
#include "mesh.hpp"
#include "mlp.hpp"
#include "setup_device.hpp"
#include "solver.hpp"
#include "tri_setup.hpp"
#include "tri_tables.hpp"

namespace wasl_b200 {

void cuda_check(cudaError_t rc, const char *what) {
  if (rc != cudaSuccess)
    throw SolverError(WASL_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(rc));
}

double bits_to_double(unsigned long long b) {
  double d;
  std::memcpy(&d, &b, sizeof(d));
  return d;
}

void throw_device_error(unsigned long long word) {
  if (!word)
    return;
  const int code = static_cast<int>(word >> 56);
  const long long element = static_cast<long long>(word & 0xffffffffffffffULL);
  if (code == 1)
    throw SolverError(WASL_ERR_NONPHYSICAL, "simulation: Euler cell average is not physical"
                                            " (element " + std::to_string(element) + ")");
  if (code == 4)
    throw SolverError(WASL_ERR_RUNTIME, "device index check: element index " +
                                            std::to_string(element) + " out of range");
  if (code == 5)
    throw SolverError(WASL_ERR_CUDA, "learned indicator: a tensor-core wait ran out");
  throw SolverError(WASL_ERR_FLOOR, "Euler positivity limiter: cell average is below a floor"
                                    " (element " + std::to_string(element) + ")");
}

double host_cell_speed(double gamma, const double *mode0, int dimensions) {
  const double scale = 1.0 / std::sqrt(2.0);
  const double s[4] = {scale * mode0[0], scale * mode0[1], scale * mode0[2], scale * mode0[3]};
  const double inv = 1.0 / s[0];
  const double vx = s[1] * inv, vy = s[2] * inv;
  const double ke = 0.5 * (s[1] * vx + s[2] * vy);
  const double p = (gamma - 1.0) * (s[3] - ke);
  const double velocity = dimensions == 1 ? std::fabs(vx) : std::hypot(vx, vy);
  return velocity + std::sqrt(gamma * p / s[0]);
}

// dst[r][i] = src[r][index[i]] over rows x ne (gather into storage order).
__global__ void gather_columns(const double *__restrict__ src, double *__restrict__ dst, int rows,
                               std::int64_t ne, const std::int32_t *__restrict__ index) {
  const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= ne)
    return;
  const std::int64_t from = index[i];
  for (int r = 0; r < rows; ++r)
    dst[r * ne + i] = src[r * ne + from];
}

// dst[r][index[i]] = src[r][i] (scatter back to the caller's order).
__global__ void scatter_columns(const double *__restrict__ src, double *__restrict__ dst, int rows,
                                std::int64_t ne, const std::int32_t *__restrict__ index) {
  const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= ne)
    return;
  const std::int64_t to = index[i];
  for (int r = 0; r < rows; ++r)
    dst[r * ne + to] = src[r * ne + i];
}

class EulerTriSolver final : public Solver {
public:
  EulerTriSolver(const wasl_gpu_config &cfg, TriTopology &&topo, const PartBoundary *part)
      : cfg_(cfg), mesh_(std::move(topo)), p_(cfg.polynomial_order),
        M_(tri_modes(cfg.polynomial_order)) {
    if (!euler_tri_order_supported(p_))
      throw SolverError(WASL_ERR_ARGUMENT, "2D Euler: polynomial order must be 0..3");
    if (cfg.precision == WASL_MIXED && !euler_tri_mixed_supported(p_, cfg.volume_rule_order))
      throw SolverError(WASL_ERR_ARGUMENT, "2D Euler mixed form: polynomial order must be 1..3"
                                           " and the volume rule order p..p+2 (or -1,"
                                           " the symmetric rule)");
    if (cfg.precision != WASL_PLAIN_FP64 && cfg.precision != WASL_MIXED)
      throw SolverError(WASL_ERR_ARGUMENT, "unknown precision form");
    cuda_check(cudaSetDevice(cfg.device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    setup_.start();
    ne_ = mesh_.element_count;
    const std::int64_t nf = mesh_.face_count();
    const int QF = p_ + 1;
    // The mixed form stores its elements along a space-filling curve (a pure
    // relabelling: every face keeps its sides and every element its slot
    // order, so the arithmetic is unchanged); the caller's order is restored
    // at every call that takes or returns per-element data.
    relabel_ = cfg.precision == WASL_MIXED && cfg.element_order == 0 && ne_ > 1;
    if (relabel_) {
      order_ = morton_order(mesh_);
      rank_.resize(ne_);
      for (std::int64_t i = 0; i < ne_; ++i)
        rank_[order_[i]] = static_cast<std::int32_t>(i);
      d_order_.upload(order_, stream_);
    }
    setup_.lap(WASL_SETUP_ORDER);

    bool has_boundary = false;
    for (std::int64_t f = 0; f < nf; ++f)
      has_boundary |= mesh_.face_right[f] < 0;
    boundary_ = cfg.boundary_left;
    if (boundary_ != WASL_PERIODIC && boundary_ != WASL_TRANSMISSIVE)
      throw SolverError(WASL_ERR_RUNTIME, "simulation: 2D Euler boundaries must be periodic");
    // The element maps on the device, for the donor search and the limiter
    // stencil's transforms (freed when setup ends).
    DeviceArray<double> d_maps;
    if (part && boundary_ != WASL_PERIODIC)
      throw SolverError(WASL_ERR_ARGUMENT, "partition boundary: the handle must be periodic");
    const bool periodic_search = has_boundary && boundary_ == WASL_PERIODIC && !part;
    if (periodic_search || (cfg.limiting && p_ > 0))
      upload_maps(mesh_, d_maps, stream_);
    PeriodicTrace trace;
    std::vector<std::int32_t> stencil_donors;
    if (periodic_search) {
      trace = periodic_trace_device(mesh_, p_, d_maps.get(), stream_);
      stencil_donors = trace.donors;
    } else if (part) {
      trace = part_trace(mesh_, p_, *part, stencil_donors);
    }
    setup_.lap(WASL_SETUP_PERIODIC);

    TriSlots t = build_tri_slots(mesh_, boundary_ == WASL_PERIODIC && has_boundary ? &trace : nullptr,
                                 QF, M_);
    boundary_count_ = t.boundary_count;
    if (boundary_count_ > 0) {
      d_bnd_element_.upload(ids(t.bnd_element), stream_);
      d_bnd_edge_.upload(t.bnd_edge, stream_);
      d_bnd_normal_.upload(t.bnd_normal, stream_);
      d_bnd_value_.resize(static_cast<std::size_t>(4) * boundary_count_);
    }
    std::vector<std::int32_t> &donors = t.donors;
    std::vector<double> &donor_basis = t.donor_basis;
    std::vector<double> &geo = t.geo, &slot_geo = t.slot_geo, &face_normal = t.face_normal;
    std::vector<std::int32_t> &slot_nbr = t.slot_nbr, &slot_face = t.slot_face,
                              &face_right = t.face_right;
    std::vector<std::uint8_t> &slot_code = t.slot_code, &face_code = t.face_code;
    if (cfg.precision == WASL_MIXED && boundary_ == WASL_PERIODIC && boundary_count_ > 0) {
      std::vector<float> basis32;
      paired_ = pair_periodic_faces(mesh_, QF, t, basis32);
      if (paired_)
        d_basis32_.upload(basis32, stream_);
    }
    if (cfg.precision == WASL_MIXED) {
      if (cfg.mixed_kernel < 0 || cfg.mixed_kernel > 1 + euler_tri_tile_shapes())
        throw SolverError(WASL_ERR_ARGUMENT, "2D Euler mixed form: unknown kernel choice");
      tile_ok_ = boundary_count_ == 0 || boundary_ == WASL_TRANSMISSIVE || paired_;
      if (cfg.mixed_kernel >= 2 && !tile_ok_)
        throw SolverError(WASL_ERR_ARGUMENT, "2D Euler mixed form: the tile kernel needs"
                                             " transmissive or paired periodic boundaries");
      if (tile_ok_) {
        if (cfg.limiting)
          d_rough_.resize(ne_ + 1); // rough list, then its count
        const TileSlotArrays ts = build_tile_slots(mesh_, t, boundary_, QF);
        d_tile_nbr_.upload(columns(ids(ts.nbr), 3), stream_);
        d_tile_code_.upload(columns(ts.code, 3), stream_);
        d_tile_aux_.upload(columns(ts.aux, 3), stream_);
        PatchEdgeArrays pe;
        patch_ok_ = build_patch_edges(mesh_, t, boundary_, QF, pe);
        if (patch_ok_) {
          d_patch_nbr_.upload(columns(ids(pe.nbr), 3), stream_);
          d_patch_info_.upload(columns(pe.info, 3), stream_);
          d_patch_geo_.upload(columns(pe.geo, 9), stream_);
        }
      }
      if (cfg.mixed_kernel >= 2 && euler_tri_tile_is_patch(cfg.mixed_kernel - 2) && !patch_ok_)
        throw SolverError(WASL_ERR_ARGUMENT, "2D Euler mixed form: the patch kernel runs on"
                                             " conforming meshes only");
      if (cfg.mixed_kernel >= 2 && cfg.limiting && !euler_tri_tile_limits(cfg.mixed_kernel - 2))
        throw SolverError(WASL_ERR_ARGUMENT, "2D Euler mixed form: the patch kernel with the"
                                             " tensor-core volume runs without the limiter");
      d_face_left_.upload(ids(mesh_.face_left), stream_);
      d_face_right_.upload(ids(face_right), stream_);
      d_face_code_.upload(face_code, stream_);
      d_face_normal_.upload(face_normal, stream_);
      d_slot_face_.upload(columns(slot_face, 3), stream_);
      d_face_record_.resize(euler_tri_mixed_face_record_bytes(p_) * nf);
    }
    d_geo_.upload(columns(geo, 5), stream_);
    d_slot_nbr_.upload(columns(ids(slot_nbr), 3), stream_);
    d_slot_code_.upload(columns(slot_code, 3), stream_);
    d_slot_geo_.upload(columns(slot_geo, 9), stream_);
    if (!donors.empty()) {
      d_donor_.upload(ids(donors), stream_);
      d_donor_basis_.upload(donor_basis, stream_);
    }
    mixed_ = cfg.precision == WASL_MIXED;
    if (mixed_ && cfg.mixed_kernel >= 1)
      kernel_ = cfg.mixed_kernel - 1;
    if (mixed_)
      upload_euler_tri_tables_mixed(p_, cfg.volume_rule_order);
    else
      upload_euler_tri_tables_f64(p_);
    std::vector<unsigned char> table(euler_tri_face_table_bytes(p_, mixed_));
    fill_euler_tri_face_table(p_, mixed_, table.data());
    d_face_table_.upload(table, stream_);
    std::vector<unsigned char> table64(euler_tri_face_table_bytes(p_, false));
    fill_euler_tri_face_table(p_, false, table64.data());
    d_face_table64_.upload(table64, stream_);
    setup_.lap(WASL_SETUP_FACES);

    limiting_ = cfg.limiting && p_ > 0;
    if (limiting_) {
      stencil_ = triangle_stencil(mesh_, p_, stencil_donors, /*transforms=*/false);
      d_neighbors_.upload(blocks(ids(stencil_.neighbors), 3), stream_);
      d_transforms_.resize(static_cast<std::size_t>(ne_) * 3 * M_ * M_);
      stencil_transforms_device(mesh_, p_, stencil_.neighbors, order_, d_maps.get(),
                                d_transforms_.get(), stream_);
      d_normal_x_.upload(columns(stencil_.normal_x, 1), stream_);
      d_normal_y_.upload(columns(stencil_.normal_y, 1), stream_);
      d_check_.upload(stencil_.check_basis, stream_);
      d_check_bound_.upload(positivity_check_bound(stencil_.check_basis, M_), stream_);
      d_limited_.resize(static_cast<std::size_t>(ne_) * 4 * M_);
      d_troubled_.resize(ne_);
    }
    setup_.lap(WASL_SETUP_STENCIL);
    d_flags_.resize(3 * ne_);
    cuda_check(cudaMemsetAsync(d_flags_.get(), 0, 3 * ne_, stream_), "memset");
    d_count_.resize(4);
    for (auto *b : {&d_u_, &d_e_, &d_s_})
      b->resize(static_cast<std::size_t>(4) * M_ * ne_);
    cuda_check(cudaMemsetAsync(d_u_.get(), 0, d_u_.size() * sizeof(double), stream_), "memset");
    d_error_.resize(1);
    d_speed_.resize(1);
    d_cfl_.resize(kCflResultWords);
    d_dt_.resize(1);
    cuda_check(cudaMemsetAsync(d_error_.get(), 0, sizeof(unsigned long long), stream_), "memset");
    length_ = minimum_altitude(mesh_);
    cuda_check(cudaStreamSynchronize(stream_), "setup");
    setup_.lap(WASL_SETUP_OTHER);
  }

  ~EulerTriSolver() override {
    if (stream_)
      cudaStreamDestroy(stream_);
  }

  std::int64_t elements() const override { return ne_; }
  std::int64_t faces() const override { return mesh_.face_count(); }
  int modes() const override { return M_; }
  int variables() const override { return 4; }
  double *state_device() override { return d_u_.get(); }

  void vertices(double *out) const override {
    for (std::int64_t e = 0; e < ne_; ++e) {
      const TriMap &m = mesh_.maps[e];
      const double v[6] = {m.x0, m.y0, m.x1, m.y1, m.x2, m.y2};
      std::memcpy(out + 6 * e, v, sizeof(v));
    }
  }

  int rule_points(int rule_order) const override { return (rule_order + 1) * (rule_order + 1); }

  void quadrature(int rule_order, double *x, double *y, double *w) const override {
    tri_quadrature(mesh_, rule_order, x, y, w);
  }

  void project(int rule_order, const double *values) override {
    set_state(tri_project(mesh_, p_, 4, rule_order, values).data());
  }

  void evaluate(int rule_order, double *values) override {
    std::vector<double> c(static_cast<std::size_t>(4) * M_ * ne_);
    get_state(c.data());
    tri_evaluate(mesh_, p_, 4, rule_order, c.data(), values);
  }

  void set_state(const double *host) override {
    speed_ready_ = false;
    // Relabelled storage: the caller's columns go through the stage buffer.
    double *target = relabel_ ? d_e_.get() : d_u_.get();
    cuda_check(cudaMemcpyAsync(target, host, d_u_.size() * sizeof(double),
                               cudaMemcpyHostToDevice, stream_),
               "set_state");
    if (relabel_) {
      gather_columns<<<static_cast<unsigned>((ne_ + 255) / 256), 256, 0, stream_>>>(
          d_e_.get(), d_u_.get(), 4 * M_, ne_, d_order_.get());
      count_launches(1);
    }
    cuda_check(cudaStreamSynchronize(stream_), "set_state");
  }

  void get_state(double *host) override {
    const double *source = d_u_.get();
    if (relabel_) {
      scatter_columns<<<static_cast<unsigned>((ne_ + 255) / 256), 256, 0, stream_>>>(
          d_u_.get(), d_e_.get(), 4 * M_, ne_, d_order_.get());
      count_launches(1);
      source = d_e_.get();
    }
    cuda_check(cudaMemcpyAsync(host, source, d_u_.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "get_state");
    cuda_check(cudaStreamSynchronize(stream_), "get_state");
  }

  void stencil_transforms(double *out, std::int64_t count) override {
    const std::int64_t width = 3 * static_cast<std::int64_t>(M_) * M_;
    if (!limiting_)
      throw SolverError(WASL_ERR_ARGUMENT, "stencil transforms: the handle has no limiter");
    if (count != ne_ * width)
      throw SolverError(WASL_ERR_ARGUMENT,
                        "stencil transforms: count must be elements x 3 x modes^2");
    std::vector<double> stored(static_cast<std::size_t>(count));
    cuda_check(cudaMemcpyAsync(stored.data(), d_transforms_.get(), count * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "transforms");
    cuda_check(cudaStreamSynchronize(stream_), "transforms");
    for (std::int64_t i = 0; i < ne_; ++i)
      std::copy(stored.begin() + i * width, stored.begin() + (i + 1) * width,
                out + (relabel_ ? order_[i] : i) * width);
  }

  void periodic_trace(std::int32_t *donors, double *basis, std::int64_t points) override {
    const std::int64_t n = static_cast<std::int64_t>(d_donor_.size());
    if (n == 0)
      throw SolverError(WASL_ERR_ARGUMENT, "periodic trace: the mesh has no periodic faces");
    if (points != n)
      throw SolverError(WASL_ERR_ARGUMENT,
                        "periodic trace: points must be boundary faces x (order + 1)");
    cuda_check(cudaMemcpyAsync(donors, d_donor_.get(), n * sizeof(std::int32_t),
                               cudaMemcpyDeviceToHost, stream_),
               "donors");
    cuda_check(cudaMemcpyAsync(basis, d_donor_basis_.get(), n * M_ * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "donor basis");
    cuda_check(cudaStreamSynchronize(stream_), "periodic trace");
    if (relabel_)
      for (std::int64_t k = 0; k < n; ++k)
        donors[k] = order_[donors[k]];
  }

  void element_order(std::int64_t *order) const override {
    for (std::int64_t i = 0; i < ne_; ++i)
      order[i] = relabel_ ? order_[i] : i;
  }

  CflArgs cfl_args(double cfl) {
    CflArgs a;
    a.ne = ne_;
    a.M = M_;
    a.dimensions = 2;
    a.state = d_u_.get();
    a.gamma = cfg_.heat_capacity_ratio;
    a.cfl = cfl;
    a.length = length_;
    a.p = p_;
    a.result = d_cfl_.get();
    a.dt = d_dt_.get();
    a.error = d_error_.get();
    a.order = relabel_ ? d_order_.get() : nullptr;
    return a;
  }

  double stable_dt(double cfl) override {
    double speed = 0.0, length = 0.0;
    cfl_parts(speed, length);
    return dt_from_parts(cfl, speed, length);
  }

  double dt_from_parts(double cfl, double speed, double length) const override {
    return speed > 0.0 ? cfl * length / (speed * (2 * p_ + 1)) : 0.0;
  }

  void cfl_parts(double &speed, double &length) override {
    CflArgs c = cfl_args(1.0);
    c.dt = nullptr; // the host forms dt
    launch_cfl(c, stream_);
    count_launches(1);
    cuda_check(cudaMemcpyAsync(scratch_.words, d_cfl_.get(), 8 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, stream_),
               "cfl result");
    cuda_check(cudaMemcpyAsync(scratch_.words + 8, d_error_.get(), sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, stream_),
               "cfl error");
    cuda_check(cudaStreamSynchronize(stream_), "cfl");
    raise_device_error(scratch_.words[8]);
    double mode0[4];
    for (int v = 0; v < 4; ++v)
      mode0[v] = bits_to_double(scratch_.words[2 + v]);
    speed = host_cell_speed(cfg_.heat_capacity_ratio, mode0, 2);
    length = length_;
  }

  void step(double dt) override {
    speed_ready_ = false;
    enqueue_step(nullptr, dt);
    if (limiting_)
      check_error();
  }

  void limit() override {
    speed_ready_ = false;
    if (!limiting_)
      return;
    cuda_check(cudaMemsetAsync(d_count_.get(), 0, sizeof(std::int32_t), stream_), "count");
    SenseArgs sa;
    sa.ne = ne_;
    sa.state = d_u_.get();
    sa.threshold = cfg_.sensor_threshold;
    sa.highest_degree_begin = stencil_.highest_degree_begin;
    sa.flags = d_flags_.get();
    sa.troubled = d_troubled_.get();
    sa.troubled_count = d_count_.get();
    launch_sense_f64(M_, sa, stream_);
    launch_limit_f64(M_, 3, limit_args(d_u_.get(), d_flags_.get()), stream_);
    count_launches(cfg_.positivity_all ? 4 : 3);
    check_error();
  }

  // Device-resident steps: dt from the largest cell-average wave speed
  // (cfl_max, then dt_from_speed, which also zeroes the speed word).  With
  // the tile kernel and no limiter, the last stage of each step also reduces
  // the next step's CFL speed, so a step after the first needs only the
  // small dt kernel and no pass over the state.
  void advance(double cfl, std::int64_t steps) override {
    for (std::int64_t n = 0; n < steps; ++n) {
      if (!speed_ready_) {
        // The speed alone: the device dt needs no arg-max (that serves the
        // host's bit-consistent stable_dt).
        CflArgs c = cfl_args(cfl);
        c.result = d_speed_.get();
        c.dt = nullptr;
        launch_cfl_speed(c, stream_);
        count_launches(1);
      }
      launch_dt_from_speed(1, d_speed_.get(), cfl, nullptr, nullptr, length_, p_, d_dt_.get(),
                           nullptr, nullptr, stream_, true);
      count_launches(1);
      fused_speed_ = mixed_ && !limiting_;
      enqueue_step(d_dt_.get(), 0.0);
      speed_ready_ = fused_speed_ && kernel_ >= 1;
      fused_speed_ = false;
    }
    cuda_check(cudaGetLastError(), "advance");
  }

  void sync() override { check_error(); }

  int indicator_features() const override {
    return limiting_ ? mlp_features_for_modes(M_) : 0;
  }

  void set_indicator(const float *weights, std::int64_t count, double lo, double hi) override {
    if (!limiting_)
      throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: needs limiting on and p >= 1");
    const MlpShape sh = mlp_shape(mlp_features_for_modes(M_));
    if (count != sh.count)
      throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: expected " +
                                               std::to_string(sh.count) + " weights");
    if (!(lo <= hi))
      throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: need lo <= hi");
    d_mlp_.upload(std::vector<float>(weights, weights + count), stream_);
    d_mlp_records_.resize(kMlpRecordBytes * ne_);
    d_mlp_stats_.resize(6);
    cuda_check(cudaMemsetAsync(d_mlp_stats_.get(), 0, 6 * sizeof(unsigned long long), stream_),
               "stats");
    mlp_lo_ = lo;
    mlp_hi_ = hi;
    cuda_check(cudaStreamSynchronize(stream_), "set indicator");
  }

  void indicator_data(float *features, std::uint8_t *labels) override {
    if (!limiting_)
      throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: needs limiting on and p >= 1");
    const int F = mlp_features_for_modes(M_);
    DeviceArray<float> f(static_cast<std::size_t>(ne_) * F);
    DeviceArray<std::uint8_t> y(ne_);
    launch_mlp_features(d_u_.get(), ne_, M_, d_neighbors_.get(), F, cfg_.sensor_threshold,
                        stencil_.highest_degree_begin, f.get(), y.get(), stream_);
    std::vector<float> fs(relabel_ ? f.size() : 0);
    std::vector<std::uint8_t> ys(relabel_ ? ne_ : 0);
    cuda_check(cudaMemcpyAsync(relabel_ ? fs.data() : features, f.get(), sizeof(float) * f.size(),
                               cudaMemcpyDeviceToHost, stream_),
               "features");
    cuda_check(cudaMemcpyAsync(relabel_ ? ys.data() : labels, y.get(), ne_,
                               cudaMemcpyDeviceToHost, stream_),
               "labels");
    cuda_check(cudaStreamSynchronize(stream_), "indicator data");
    if (relabel_)
      for (std::int64_t i = 0; i < ne_; ++i) {
        std::copy(fs.begin() + i * F, fs.begin() + (i + 1) * F,
                  features + static_cast<std::int64_t>(order_[i]) * F);
        labels[order_[i]] = ys[i];
      }
  }

  // The network's logits for the current state, from the inference kernel
  // (its flags and troubled list go to scratch; the state is untouched).
  void indicator_logits(float *logits) override {
    if (d_mlp_.size() == 0)
      throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: not set");
    DeviceArray<float> z(ne_);
    DeviceArray<std::uint8_t> flags(ne_);
    DeviceArray<std::int32_t> list(ne_ + 1);
    cuda_check(cudaMemsetAsync(list.get() + ne_, 0, sizeof(std::int32_t), stream_), "count");
    MlpIndicatorArgs m;
    m.shape = mlp_shape(mlp_features_for_modes(M_));
    m.params = d_mlp_.get();
    m.lo = static_cast<float>(mlp_lo_);
    m.hi = static_cast<float>(mlp_hi_);
    m.state = d_u_.get();
    m.ne = ne_;
    m.M = M_;
    m.neighbors = d_neighbors_.get();
    m.threshold = cfg_.sensor_threshold;
    m.highest_degree_begin = stencil_.highest_degree_begin;
    m.flags = flags.get();
    m.troubled = list.get();
    m.troubled_count = list.get() + ne_;
    m.logits = z.get();
    m.records = d_mlp_records_.get();
    m.error = d_error_.get();
    m.kernel = mlp_kernel_;
    launch_mlp_indicator(m, stream_);
    std::vector<float> zs(relabel_ ? ne_ : 0);
    cuda_check(cudaMemcpyAsync(relabel_ ? zs.data() : logits, z.get(), sizeof(float) * ne_,
                               cudaMemcpyDeviceToHost, stream_),
               "logits");
    cuda_check(cudaStreamSynchronize(stream_), "indicator logits");
    if (relabel_)
      for (std::int64_t i = 0; i < ne_; ++i)
        logits[order_[i]] = zs[i];
  }

  void set_indicator_kernel(int kernel) override {
    if (kernel != 0 && kernel != 1)
      throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: kernel must be 0 (tcgen05) or 1"
                                           " (mma.sync)");
    mlp_kernel_ = kernel;
  }

  void indicator_stats(unsigned long long *stats, bool reset) override {
    if (d_mlp_.size() == 0)
      throw SolverError(WASL_ERR_ARGUMENT, "learned indicator: not set");
    cuda_check(cudaMemcpyAsync(stats, d_mlp_stats_.get(), 6 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, stream_),
               "stats");
    if (reset)
      cuda_check(cudaMemsetAsync(d_mlp_stats_.get(), 0, 6 * sizeof(unsigned long long), stream_),
                 "stats");
    cuda_check(cudaStreamSynchronize(stream_), "stats");
  }

  int kernel_choice(double *ms, int capacity, int &count) override {
    count = static_cast<int>(tuning_.ms.size());
    for (int i = 0; i < count && i < capacity; ++i)
      ms[i] = tuning_.ms[i];
    return mixed_ ? kernel_ : -1;
  }

  void flags(std::uint8_t *out) override {
    std::vector<std::uint8_t> stored(relabel_ ? 3 * ne_ : 0);
    cuda_check(cudaMemcpyAsync(relabel_ ? stored.data() : out, d_flags_.get(), 3 * ne_,
                               cudaMemcpyDeviceToHost, stream_),
               "flags");
    cuda_check(cudaStreamSynchronize(stream_), "flags");
    if (relabel_)
      for (int k = 0; k < 3; ++k)
        for (std::int64_t i = 0; i < ne_; ++i)
          out[k * ne_ + order_[i]] = stored[k * ne_ + i];
  }

  void mass_energy(double &mass, double &energy) override {
    std::vector<double> rho(ne_), en(ne_);
    cuda_check(cudaMemcpyAsync(rho.data(), d_u_.get(), ne_ * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "mass");
    cuda_check(cudaMemcpyAsync(en.data(), d_u_.get() + static_cast<std::size_t>(3) * M_ * ne_,
                               ne_ * sizeof(double), cudaMemcpyDeviceToHost, stream_),
               "energy");
    cuda_check(cudaStreamSynchronize(stream_), "mass");
    mass = energy = 0.0;
    for (std::int64_t e = 0; e < ne_; ++e) {
      const double w = std::sqrt(2.0) * mesh_.maps[relabel_ ? order_[e] : e].jacobian_determinant();
      mass += w * rho[e];
      energy += w * en[e];
    }
  }

private:
  // One step with dt read from device memory (dt_device, written by the CFL
  // kernels) or, when dt_device is null, passed by value.
  void enqueue_step(const double *dt_device, double dt_value) {
    StageArgs a;
    a.mesh.ne = ne_;
    a.mesh.geo = d_geo_.get();
    a.mesh.slot_nbr = d_slot_nbr_.get();
    a.mesh.slot_code = d_slot_code_.get();
    a.mesh.slot_geo = d_slot_geo_.get();
    a.mesh.donor = d_donor_.get();
    a.mesh.donor_basis = d_donor_basis_.get();
    a.mesh.boundary = boundary_;
    a.boundary.count = boundary_count_;
    a.boundary.element = d_bnd_element_.get();
    a.boundary.local_edge = d_bnd_edge_.get();
    a.boundary.normal = d_bnd_normal_.get();
    a.boundary.value = d_bnd_value_.get();
    a.boundary.paired = paired_ ? 1 : 0;
    a.boundary.basis32 = d_basis32_.get();
    a.faces.count = mesh_.face_count();
    a.faces.left = d_face_left_.get();
    a.faces.right = d_face_right_.get();
    a.faces.code = d_face_code_.get();
    a.faces.normal = d_face_normal_.get();
    a.faces.record = d_face_record_.get();
    a.faces.slot_face = d_slot_face_.get();
    a.face_table = d_face_table_.get();
    a.face_table64 = d_face_table64_.get();
    a.tile.nbr = d_tile_nbr_.get();
    a.tile.code = d_tile_code_.get();
    a.tile.aux = d_tile_aux_.get();
    a.patch.nbr = d_patch_nbr_.get();
    a.patch.info = d_patch_info_.get();
    a.patch.geo = d_patch_geo_.get();
    // FP64 face islands at discontinuities (the rough pass), with the limiter.
    a.rough = limiting_ ? d_rough_.get() : nullptr;
    a.rough_count = a.rough ? d_rough_.get() + ne_ : nullptr;
    a.dt = dt_device;
    a.dt_value = dt_value;
    a.gamma = cfg_.heat_capacity_ratio;
    const bool learned = limiting_ && d_mlp_.size() > 0;
    a.sense = limiting_ && !learned ? 1 : 0;
    a.threshold = cfg_.sensor_threshold;
    a.highest_degree_begin = stencil_.highest_degree_begin;
    a.troubled = d_troubled_.get();
    a.troubled_count = d_count_.get();
    if (mixed_ && kernel_ < 0)
      tune_mixed(a);
    double *ins[3] = {d_u_.get(), d_e_.get(), d_s_.get()};
    double *outs[3] = {d_e_.get(), d_s_.get(), d_u_.get()};
    for (int k = 0; k < 3; ++k) {
      a.stage = k;
      a.in = ins[k];
      a.u0 = d_u_.get();
      a.out = outs[k];
      a.flags = d_flags_.get() + k * ne_;
      if (limiting_)
        cuda_check(cudaMemsetAsync(d_count_.get(), 0, sizeof(std::int32_t), stream_), "count");
      a.speed_max = fused_speed_ && k == 2 && kernel_ >= 1 ? d_speed_.get() : nullptr;
      a.error = d_error_.get();
      stage_begin();
      if (mixed_)
        launch_mixed(a);
      else {
        launch_euler_tri_stage_f64(p_, a, stream_);
        count_launches(1);
      }
      stage_end();
      if (learned) {
        MlpIndicatorArgs m;
        m.shape = mlp_shape(mlp_features_for_modes(M_));
        m.params = d_mlp_.get();
        m.lo = static_cast<float>(mlp_lo_);
        m.hi = static_cast<float>(mlp_hi_);
        m.state = outs[k];
        m.ne = ne_;
        m.M = M_;
        m.neighbors = d_neighbors_.get();
        m.threshold = cfg_.sensor_threshold;
        m.highest_degree_begin = stencil_.highest_degree_begin;
        m.flags = d_flags_.get() + k * ne_;
        m.troubled = d_troubled_.get();
        m.troubled_count = d_count_.get();
        m.stats = d_mlp_stats_.get();
        m.records = d_mlp_records_.get();
        m.error = d_error_.get();
        m.kernel = mlp_kernel_;
        launch_mlp_indicator(m, stream_);
        count_launches(2);
      }
      if (limiting_) {
        launch_limit_f64(M_, 3, limit_args(outs[k], d_flags_.get() + k * ne_), stream_);
        count_launches(cfg_.positivity_all ? 3 : 2);
      }
    }
    cuda_check(cudaGetLastError(), "stage launch");
  }

  // kernel_: 0 face-centric kernels, 1 + s the tile kernel in shape s.
  void launch_mixed(const StageArgs &a) {
    if (kernel_ == 0) {
      launch_euler_tri_stage_mixed(p_, cfg_.volume_rule_order, a, stream_);
      count_launches(boundary_count_ > 0 && boundary_ != WASL_TRANSMISSIVE && !paired_ ? 3 : 2);
    } else {
      launch_euler_tri_stage_tile(p_, cfg_.volume_rule_order, kernel_ - 1, a, stream_);
      count_launches(a.rough ? 2 : 1);
    }
  }

  // Times every kernel choice on the three stages of a step of the current
  // state into scratch (u^n is read, not written; sensing off) and keeps the
  // fastest, per polynomial order, rule order and mesh size class.
  void tune_mixed(StageArgs a) {
    // With the limiter (flows with discontinuities) only the tile kernel,
    // whose second pass evaluates faces at discontinuities in FP64, competes;
    // the patch kernel's shapes only where its edge arrays were built.
    const int base = tile_ok_ && limiting_ ? 1 : 0;
    std::vector<int> kernels; // kernel_ values: 0 face-centric, 1 + shape
    if (!base)
      kernels.push_back(0);
    if (tile_ok_)
      for (int sh = 0; sh < euler_tri_tile_shapes(); ++sh)
        if ((!euler_tri_tile_is_patch(sh) || patch_ok_) &&
            (!limiting_ || euler_tri_tile_limits(sh)))
          kernels.push_back(1 + sh);
    // Each variant runs the three stages of a step on the current state, into
    // the stage buffers only (the last stage writes the first stage buffer
    // instead of u^n), so the stages that also read u^n weigh in.
    a.u0 = d_u_.get();
    a.sense = 0;
    a.dt = nullptr;
    a.dt_value = 0.0;
    double *ins[3] = {d_u_.get(), d_e_.get(), d_s_.get()};
    double *outs[3] = {d_e_.get(), d_s_.get(), d_e_.get()};
    const std::string key = "euler_tri_mixed/p" + std::to_string(p_) + "/rule" +
                            std::to_string(cfg_.volume_rule_order ? cfg_.volume_rule_order : p_ + 2) +
                            "/bnd" + std::to_string(boundary_count_ > 0 ? boundary_ : -1) +
                            "/size" + std::to_string(size_class(ne_));
    const TuneResult timed = autotune(key + (base ? "/tile-only" : ""),
                                      static_cast<int>(kernels.size()), [&](int i) {
      kernel_ = kernels[i];
      for (int k = 0; k < 3; ++k) {
        a.stage = k;
        a.in = ins[k];
        a.out = outs[k];
        launch_mixed(a);
      }
    }, stream_);
    // Per stage, by kernel value (0 for the variants not timed).
    tuning_.ms.assign(1 + euler_tri_tile_shapes(), 0.0);
    for (std::size_t i = 0; i < kernels.size(); ++i)
      tuning_.ms[kernels[i]] = timed.ms[i] / 3.0;
    kernel_ = kernels[timed.choice];
    tuning_.choice = kernel_;
  }

  // Per-element host arrays [count][ne] in storage order.
  template <typename T> std::vector<T> columns(const std::vector<T> &v, int count) const {
    if (!relabel_)
      return v;
    std::vector<T> out(v.size());
    for (int r = 0; r < count; ++r)
      for (std::int64_t i = 0; i < ne_; ++i)
        out[r * ne_ + i] = v[r * ne_ + order_[i]];
    return out;
  }
  // Per-element host arrays [ne][width] in storage order.
  template <typename T> std::vector<T> blocks(const std::vector<T> &v, std::int64_t width) const {
    if (!relabel_)
      return v;
    std::vector<T> out(v.size());
    for (std::int64_t i = 0; i < ne_; ++i)
      std::copy(v.begin() + order_[i] * width, v.begin() + (order_[i] + 1) * width,
                out.begin() + i * width);
    return out;
  }
  // Element indices (>= 0) relabelled; negative codes kept.
  std::vector<std::int32_t> ids(std::vector<std::int32_t> v) const {
    if (relabel_)
      for (auto &x : v)
        if (x >= 0)
          x = rank_[x];
    return v;
  }

  LimitArgs limit_args(double *state, const std::uint8_t *flags) {
    LimitArgs l;
    l.positivity_all = cfg_.positivity_all ? 1 : 0;
    l.flags = flags;
    l.relative_floor = mixed_ ? kMixedRelativeFloor : 0.0;
    l.check_bound = d_check_bound_.get();
    l.ne = ne_;
    l.state = state;
    l.troubled = d_troubled_.get();
    l.troubled_count = d_count_.get();
    l.neighbors = d_neighbors_.get();
    l.transforms = d_transforms_.get();
    l.normal_x = d_normal_x_.get();
    l.normal_y = d_normal_y_.get();
    l.check_basis = d_check_.get();
    l.check_points = stencil_.check_point_count();
    l.gamma = cfg_.heat_capacity_ratio;
    l.density_floor = cfg_.density_floor;
    l.pressure_floor = cfg_.pressure_floor;
    l.limited = d_limited_.get();
    l.error = d_error_.get();
    return l;
  }

  void check_error() {
    cuda_check(cudaMemcpyAsync(scratch_.words + 8, d_error_.get(), sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, stream_),
               "error word");
    cuda_check(cudaStreamSynchronize(stream_), "step");
    raise_device_error(scratch_.words[8]);
  }

  void raise_device_error(unsigned long long word) {
    if (!word)
      return;
    cuda_check(cudaMemsetAsync(d_error_.get(), 0, sizeof(unsigned long long), stream_), "memset");
    throw_device_error(word);
  }

  wasl_gpu_config cfg_;
  TriTopology mesh_;
  int p_, M_;
  std::int64_t ne_ = 0;
  int boundary_ = 0;
  std::int64_t boundary_count_ = 0;
  bool limiting_ = false;
  bool mixed_ = false;
  bool paired_ = false;
  bool tile_ok_ = false;
  bool relabel_ = false;  // elements stored along a space-filling curve
  std::vector<std::int32_t> order_, rank_; // storage -> caller, caller -> storage
  DeviceArray<std::int32_t> d_order_;
  bool patch_ok_ = false; // the patch kernel's edge arrays exist
  DeviceArray<std::int32_t> d_patch_nbr_;
  DeviceArray<std::uint8_t> d_patch_info_;
  DeviceArray<double> d_patch_geo_;
  bool fused_speed_ = false; // this step's last stage reduces the next CFL speed
  bool speed_ready_ = false; // d_speed_ holds the current state's CFL speed
  DeviceArray<unsigned long long> d_speed_;
  int kernel_ = -1; // mixed form: -1 not chosen yet, 0 face-centric, 1 + s tile shape s
  TuneResult tuning_;
  DeviceArray<std::int32_t> d_tile_nbr_, d_tile_aux_, d_rough_;
  DeviceArray<float> d_mlp_; // learned indicator weights (empty: the reference sensor)
  DeviceArray<double> d_check_bound_;
  DeviceArray<unsigned long long> d_mlp_stats_;
  DeviceArray<unsigned char> d_mlp_records_; // per-element inference records
  double mlp_lo_ = 0.1, mlp_hi_ = 0.9;
  int mlp_kernel_ = 0; // inference: 0 tcgen05 MMAs, 1 mma.sync
  DeviceArray<std::uint8_t> d_tile_code_;
  DeviceArray<float> d_basis32_;
  double length_ = 0.0;
  LimiterStencil stencil_;
  PinnedScratch scratch_;
  DeviceArray<double> d_bnd_normal_, d_bnd_value_, d_face_normal_;
  DeviceArray<std::int32_t> d_face_left_, d_face_right_, d_slot_face_;
  DeviceArray<std::uint8_t> d_face_code_;
  DeviceArray<unsigned char> d_face_record_;
  DeviceArray<std::int32_t> d_bnd_element_;
  DeviceArray<std::uint8_t> d_bnd_edge_;
  DeviceArray<double> d_geo_, d_slot_geo_, d_donor_basis_, d_transforms_, d_normal_x_,
      d_normal_y_, d_check_, d_limited_, d_u_, d_e_, d_s_, d_dt_;
  DeviceArray<std::int32_t> d_slot_nbr_, d_donor_, d_neighbors_, d_troubled_, d_count_;
  DeviceArray<std::uint8_t> d_slot_code_, d_flags_;
  DeviceArray<unsigned char> d_face_table_, d_face_table64_;
  DeviceArray<unsigned long long> d_error_, d_cfl_;
};

std::unique_ptr<Solver> make_euler_tri_solver(const wasl_gpu_config &cfg, TriTopology &&topo,
                                              const PartBoundary *part) {
  return std::make_unique<EulerTriSolver>(cfg, std::move(topo), part);
}

} // namespace wasl_b200
