// 1D solvers on line meshes: compressible Euler with the stage limiter, and
// scalar advection.  Mirrors the reference case drivers:
//   Euler  cpp/src/case/euler_line.cpp:14-46 (limiter stencil with periodic or
//          open ends, CFL from the state each step, cfl_timestep.cpp:70-76)
//   scalar cpp/src/case/scalar_advection_line.cpp:11-33 (CFL step fixed at
//          setup, cfl_timestep.cpp:55-60; no limiter)
// Elements are stored in the reference's order (sorted left to right), the
// state as [variable][mode][element] (the checkpoint layout; for the scalar
// solver [mode][element], the transpose of the reference's solver layout,
// cpp/src/case/scalar_coefficient_layout.cpp).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "basis.hpp"
#include "kernels.hpp"
#include "mesh.hpp"
#include "solver.hpp"

namespace wasl_b200 {

class LineSolver final : public Solver {
public:
  LineSolver(const wasl_gpu_config &cfg, LineTopology &&topo)
      : cfg_(cfg), mesh_(std::move(topo)), p_(cfg.polynomial_order), M_(line_modes(p_)),
        V_(cfg.equation == WASL_EULER ? 4 : 1) {
    if (!line_order_supported(p_))
      throw SolverError(WASL_ERR_ARGUMENT, "line polynomial order must be 0..6");
    if (cfg.precision != WASL_PLAIN_FP64)
      throw SolverError(WASL_ERR_ARGUMENT, "line meshes: only the plain FP64 form");
    left_kind_ = end_kind(cfg.boundary_left);
    right_kind_ = end_kind(cfg.boundary_right);
    if ((left_kind_ == WASL_PERIODIC) != (right_kind_ == WASL_PERIODIC))
      throw SolverError(WASL_ERR_RUNTIME,
                        "boundaries: periodic conditions must be applied to both line ends");
    if (V_ == 4 && (left_kind_ == WASL_INFLOW || right_kind_ == WASL_INFLOW))
      throw SolverError(WASL_ERR_ARGUMENT, "line Euler exterior: inflow is not implemented");
    cuda_check(cudaSetDevice(cfg.device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    ne_ = mesh_.element_count;

    std::vector<double> inv(ne_);
    for (std::int64_t e = 0; e < ne_; ++e)
      inv[e] = 1.0 / ((mesh_.x_right[e] - mesh_.x_left[e]) / 2.0);
    d_inv_jacobian_.upload(inv, stream_);
    fill_line_table(p_, V_ == 4 ? p_ + 1 : std::max(1, p_), table_);

    limiting_ = V_ == 4 && cfg.limiting && p_ > 0;
    if (limiting_) {
      stencil_ = line_stencil(mesh_, p_, left_kind_ == WASL_PERIODIC);
      d_neighbors_.upload(stencil_.neighbors, stream_);
      d_transforms_.upload(stencil_.transforms, stream_);
      d_normal_x_.upload(stencil_.normal_x, stream_);
      d_normal_y_.upload(stencil_.normal_y, stream_);
      d_check_.upload(stencil_.check_basis, stream_);
      d_limited_.resize(static_cast<std::size_t>(ne_) * 4 * M_);
      d_troubled_.resize(ne_);
    }
    d_flags_.resize(3 * ne_);
    cuda_check(cudaMemsetAsync(d_flags_.get(), 0, 3 * ne_, stream_), "memset");
    d_count_.resize(4);
    for (auto *b : {&d_u_, &d_e_, &d_s_})
      b->resize(static_cast<std::size_t>(V_) * M_ * ne_);
    cuda_check(cudaMemsetAsync(d_u_.get(), 0, d_u_.size() * sizeof(double), stream_), "memset");
    d_error_.resize(1);
    d_cfl_.resize(kCflResultWords);
    d_dt_.resize(1);
    cuda_check(cudaMemsetAsync(d_error_.get(), 0, sizeof(unsigned long long), stream_), "memset");
    length_ = minimum_length(mesh_);
    cuda_check(cudaStreamSynchronize(stream_), "setup");
  }

  ~LineSolver() override {
    if (stream_)
      cudaStreamDestroy(stream_);
  }

  std::int64_t elements() const override { return ne_; }
  std::int64_t faces() const override { return mesh_.face_count(); }
  int modes() const override { return M_; }
  int variables() const override { return V_; }
  double *state_device() override { return d_u_.get(); }

  void vertices(double *out) const override {
    for (std::int64_t e = 0; e < ne_; ++e) {
      out[2 * e] = mesh_.x_left[e];
      out[2 * e + 1] = mesh_.x_right[e];
    }
  }

  // The (r+1)-point Gauss rule.
  int rule_points(int rule_order) const override { return rule_order + 1; }

  void quadrature(int rule_order, double *x, double *y, double *w) const override {
    const Rule1D rule = gauss_legendre(rule_order + 1);
    const int Q = rule_order + 1;
    for (std::int64_t e = 0; e < ne_; ++e) {
      const double xl = mesh_.x_left[e], xr = mesh_.x_right[e];
      const double centre = (xl + xr) / 2.0, jac = (xr - xl) / 2.0;
      for (int q = 0; q < Q; ++q) {
        x[e * Q + q] = centre + jac * rule.x[q];
        if (y)
          y[e * Q + q] = 0.0;
        if (w)
          w[e * Q + q] = rule.w[q] * std::fabs(jac);
      }
    }
  }

  // cpp/include/wasl/dg/l2_projection.hpp:36-53
  void project(int rule_order, const double *values) override {
    const Rule1D rule = gauss_legendre(rule_order + 1);
    const int Q = rule_order + 1;
    std::vector<std::vector<double>> basis(Q);
    for (int q = 0; q < Q; ++q)
      basis[q] = legendre(rule.x[q], p_);
    std::vector<double> c(static_cast<std::size_t>(V_) * M_ * ne_, 0.0);
    for (std::int64_t e = 0; e < ne_; ++e)
      for (int q = 0; q < Q; ++q) {
        const double *val = values + (e * Q + q) * V_;
        for (int v = 0; v < V_; ++v)
          for (int m = 0; m < M_; ++m)
            c[(static_cast<std::int64_t>(v) * M_ + m) * ne_ + e] += rule.w[q] * val[v] * basis[q][m];
      }
    set_state(c.data());
  }

  void evaluate(int rule_order, double *values) override {
    const Rule1D rule = gauss_legendre(rule_order + 1);
    const int Q = rule_order + 1;
    std::vector<double> c(static_cast<std::size_t>(V_) * M_ * ne_);
    get_state(c.data());
    std::vector<std::vector<double>> basis(Q);
    for (int q = 0; q < Q; ++q)
      basis[q] = legendre(rule.x[q], p_);
    for (std::int64_t e = 0; e < ne_; ++e)
      for (int q = 0; q < Q; ++q)
        for (int v = 0; v < V_; ++v) {
          double s = 0.0;
          for (int m = 0; m < M_; ++m)
            s += c[(static_cast<std::int64_t>(v) * M_ + m) * ne_ + e] * basis[q][m];
          values[(e * Q + q) * V_ + v] = s;
        }
  }

  void set_state(const double *host) override {
    cuda_check(cudaMemcpyAsync(d_u_.get(), host, d_u_.size() * sizeof(double),
                               cudaMemcpyHostToDevice, stream_),
               "set_state");
    cuda_check(cudaStreamSynchronize(stream_), "set_state");
  }

  void get_state(double *host) override {
    cuda_check(cudaMemcpyAsync(host, d_u_.get(), d_u_.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "get_state");
    cuda_check(cudaStreamSynchronize(stream_), "get_state");
  }

  double stable_dt(double cfl) override {
    if (V_ == 1) {
      // advection_cfl_timestep: fixed by the mesh and the wavespeed.
      if (ne_ == 0 || cfg_.velocity_x == 0.0)
        return 0.0;
      return cfl * length_ / (std::fabs(cfg_.velocity_x) * (2.0 * p_ + 1.0));
    }
    launch_cfl(cfl_args(cfl), stream_);
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
    const double speed = host_cell_speed(cfg_.heat_capacity_ratio, mode0, 1);
    return speed > 0.0 ? cfl * length_ / (speed * (2 * p_ + 1)) : 0.0;
  }

  void step(double dt) override {
    enqueue_step(nullptr, dt);
    if (limiting_)
      check_error();
  }

  void limit() override {
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
    launch_limit_f64(M_, 2, limit_args(d_u_.get()), stream_);
    count_launches(3);
    check_error();
  }

  void advance(double cfl, std::int64_t steps) override {
    if (V_ == 1) {
      const double dt = stable_dt(cfl);
      for (std::int64_t n = 0; n < steps; ++n)
        enqueue_step(nullptr, dt);
    } else {
      for (std::int64_t n = 0; n < steps; ++n) {
        launch_cfl(cfl_args(cfl), stream_);
        count_launches(1);
        enqueue_step(d_dt_.get(), 0.0);
      }
    }
    cuda_check(cudaGetLastError(), "advance");
  }

  void sync() override { check_error(); }

  void run_resident(double cfl, double start_time, double end_time, std::uint64_t max_steps,
                    std::uint64_t &steps, double &time) override {
    if (limiting_)
      throw SolverError(WASL_ERR_ARGUMENT, "resident run: runs without the limiter only");
    if (line_run_bytes(V_, p_, ne_) > kLineRunMaxBytes)
      throw SolverError(WASL_ERR_ARGUMENT,
                        "resident run: " + std::to_string(ne_) +
                            " elements do not fit in one CTA's shared memory");
    LineRunArgs r;
    r.stage = stage_args();
    r.state = d_u_.get();
    r.fixed_dt = V_ == 1 ? stable_dt(cfl) : 0.0;
    r.cfl = cfl;
    r.length = length_;
    r.start_time = start_time;
    r.end_time = end_time;
    r.max_steps = max_steps;
    r.result = d_cfl_.get();
    r.error = d_error_.get();
    launch_line_run_f64(V_, p_, r, stream_);
    count_launches(1);
    cuda_check(cudaGetLastError(), "resident run");
    cuda_check(cudaMemcpyAsync(scratch_.words, d_cfl_.get(), 3 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, stream_),
               "resident run");
    check_error();
    steps = scratch_.words[0];
    time = bits_to_double(scratch_.words[1]);
    if (scratch_.words[2] == 1)
      throw SolverError(WASL_ERR_RUNTIME, "simulation: timestep cannot advance time");
  }

  void flags(std::uint8_t *out) override {
    cuda_check(cudaMemcpyAsync(out, d_flags_.get(), 3 * ne_, cudaMemcpyDeviceToHost, stream_),
               "flags");
    cuda_check(cudaStreamSynchronize(stream_), "flags");
  }

  // euler_diagnostics.cpp:26-31 / scalar_diagnostics.cpp:21-27 (scalar: energy = mass).
  void mass_energy(double &mass, double &energy) override {
    std::vector<double> rho(ne_), en(ne_);
    cuda_check(cudaMemcpyAsync(rho.data(), d_u_.get(), ne_ * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "mass");
    if (V_ == 4)
      cuda_check(cudaMemcpyAsync(en.data(), d_u_.get() + static_cast<std::size_t>(3) * M_ * ne_,
                                 ne_ * sizeof(double), cudaMemcpyDeviceToHost, stream_),
                 "energy");
    cuda_check(cudaStreamSynchronize(stream_), "mass");
    mass = energy = 0.0;
    for (std::int64_t e = 0; e < ne_; ++e) {
      const double w = std::sqrt(2.0) * ((mesh_.x_right[e] - mesh_.x_left[e]) / 2.0);
      mass += w * rho[e];
      if (V_ == 4)
        energy += w * en[e];
    }
    if (V_ == 1)
      energy = mass;
  }

private:
  // Line end kinds: periodic, inflow, outflow (transmissive is outflow).
  static int end_kind(int kind) {
    if (kind == WASL_TRANSMISSIVE)
      return WASL_OUTFLOW;
    if (kind != WASL_PERIODIC && kind != WASL_INFLOW && kind != WASL_OUTFLOW)
      throw SolverError(WASL_ERR_ARGUMENT, "boundaries: unknown line boundary kind");
    return kind;
  }

  CflArgs cfl_args(double cfl) {
    CflArgs a;
    a.ne = ne_;
    a.M = M_;
    a.dimensions = 1;
    a.state = d_u_.get();
    a.gamma = cfg_.heat_capacity_ratio;
    a.cfl = cfl;
    a.length = length_;
    a.p = p_;
    a.result = d_cfl_.get();
    a.dt = d_dt_.get();
    a.error = d_error_.get();
    return a;
  }

  // The stage arguments common to every stage (mesh, table, ends, physics).
  LineStageArgs stage_args() const {
    LineStageArgs a;
    a.ne = ne_;
    a.inv_jacobian = d_inv_jacobian_.get();
    a.gamma = cfg_.heat_capacity_ratio;
    a.speed = cfg_.velocity_x;
    a.left_kind = left_kind_;
    a.right_kind = right_kind_;
    a.left_value = cfg_.inflow_left;
    a.right_value = cfg_.inflow_right;
    a.table = table_;
    return a;
  }

  void enqueue_step(const double *dt_device, double dt_value) {
    LineStageArgs a;
    a.ne = ne_;
    a.inv_jacobian = d_inv_jacobian_.get();
    a.dt = dt_device;
    a.dt_value = dt_value;
    a.gamma = cfg_.heat_capacity_ratio;
    a.speed = cfg_.velocity_x;
    a.left_kind = left_kind_;
    a.right_kind = right_kind_;
    a.left_value = cfg_.inflow_left;
    a.right_value = cfg_.inflow_right;
    a.sense = limiting_ ? 1 : 0;
    a.threshold = cfg_.sensor_threshold;
    a.highest_degree_begin = stencil_.highest_degree_begin;
    a.troubled = d_troubled_.get();
    a.troubled_count = d_count_.get();
    a.table = table_;
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
      stage_begin();
      launch_line_stage_f64(V_, p_, a, stream_);
      stage_end();
      count_launches(1);
      if (limiting_) {
        launch_limit_f64(M_, 2, limit_args(outs[k]), stream_);
        count_launches(2);
      }
    }
    cuda_check(cudaGetLastError(), "stage launch");
  }

  LimitArgs limit_args(double *state) {
    LimitArgs l;
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
  LineTopology mesh_;
  int p_, M_, V_;
  std::int64_t ne_ = 0;
  int left_kind_ = WASL_PERIODIC, right_kind_ = WASL_PERIODIC;
  bool limiting_ = false;
  double length_ = 0.0;
  LineTable table_{};
  LimiterStencil stencil_;
  PinnedScratch scratch_;
  DeviceArray<double> d_inv_jacobian_, d_transforms_, d_normal_x_, d_normal_y_, d_check_,
      d_limited_, d_u_, d_e_, d_s_, d_dt_;
  DeviceArray<std::int32_t> d_neighbors_, d_troubled_, d_count_;
  DeviceArray<std::uint8_t> d_flags_;
  DeviceArray<unsigned long long> d_error_, d_cfl_;
};

std::unique_ptr<Solver> make_line_solver(const wasl_gpu_config &cfg, LineTopology &&topo) {
  return std::make_unique<LineSolver>(cfg, std::move(topo));
}

} // namespace wasl_b200
