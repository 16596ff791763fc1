// 2D scalar advection on triangles with periodic boundaries.  Mirrors the
// reference case driver cpp/src/case/scalar_advection_triangle.cpp:16-45:
// periodic trace once, CFL step fixed at setup (cfl_timestep.cpp:62-68), then
// ssp_rk3_step without a limiter.  State [mode][element] (the checkpoint
// layout; the transpose of the reference's solver layout).
#include <cmath>
#include <cstring>

#include "basis.hpp"
#include "kernels.hpp"
#include "mesh.hpp"
#include "setup_device.hpp"
#include "solver.hpp"
#include "tri_tables.hpp"

namespace wasl_b200 {

class ScalarTriSolver final : public Solver {
public:
  ScalarTriSolver(const wasl_gpu_config &cfg, TriTopology &&topo, const PartBoundary *part)
      : cfg_(cfg), mesh_(std::move(topo)), p_(cfg.polynomial_order), M_(tri_modes(p_)) {
    if (!euler_tri_order_supported(p_))
      throw SolverError(WASL_ERR_ARGUMENT, "2D scalar advection: polynomial order must be 0..3");
    if (cfg.precision != WASL_PLAIN_FP64)
      throw SolverError(WASL_ERR_ARGUMENT, "2D scalar advection: only the plain FP64 form");
    if (cfg.boundary_left != WASL_PERIODIC)
      throw SolverError(WASL_ERR_RUNTIME,
                        "simulation: 2D scalar-advection boundaries must be periodic");
    cuda_check(cudaSetDevice(cfg.device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    setup_.start();
    ne_ = mesh_.element_count;
    const int QF = p_ + 1;
    bool has_boundary = false;
    for (std::int64_t f = 0; f < mesh_.face_count(); ++f)
      has_boundary |= mesh_.face_right[f] < 0;
    PeriodicTrace trace;
    if (part) {
      std::vector<std::int32_t> stencil_donors;
      trace = part_trace(mesh_, p_, *part, stencil_donors);
    } else if (has_boundary) {
      DeviceArray<double> d_maps;
      upload_maps(mesh_, d_maps, stream_);
      trace = periodic_trace_device(mesh_, p_, d_maps.get(), stream_);
    }
    setup_.lap(WASL_SETUP_PERIODIC);
    const TriSlots t = build_tri_slots(mesh_, has_boundary ? &trace : nullptr, QF, M_);
    d_geo_.upload(t.geo, stream_);
    d_slot_nbr_.upload(t.slot_nbr, stream_);
    d_slot_code_.upload(t.slot_code, stream_);
    d_slot_geo_.upload(t.slot_geo, stream_);
    if (!t.donors.empty()) {
      d_donor_.upload(t.donors, stream_);
      d_donor_basis_.upload(t.donor_basis, stream_);
    }
    upload_scalar_tri_tables(p_);
    std::vector<unsigned char> table(euler_tri_face_table_bytes(p_, false));
    fill_euler_tri_face_table(p_, false, table.data());
    d_face_table_.upload(table, stream_);
    for (auto *b : {&d_u_, &d_e_, &d_s_})
      b->resize(static_cast<std::size_t>(M_) * ne_);
    cuda_check(cudaMemsetAsync(d_u_.get(), 0, d_u_.size() * sizeof(double), stream_), "memset");
    d_flags_.resize(3 * ne_);
    cuda_check(cudaMemsetAsync(d_flags_.get(), 0, 3 * ne_, stream_), "memset");
    length_ = minimum_altitude(mesh_);
    cuda_check(cudaStreamSynchronize(stream_), "setup");
    setup_.lap(WASL_SETUP_OTHER);
  }

  ~ScalarTriSolver() override {
    if (stream_)
      cudaStreamDestroy(stream_);
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
  }

  std::int64_t elements() const override { return ne_; }
  std::int64_t faces() const override { return mesh_.face_count(); }
  int modes() const override { return M_; }
  int variables() const override { return 1; }
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
    const Rule2D rule = triangle_rule(rule_order);
    const int Q = rule.size();
    for (std::int64_t e = 0; e < ne_; ++e) {
      const TriMap &m = mesh_.maps[e];
      const double jac = std::fabs(m.jacobian_determinant());
      for (int q = 0; q < Q; ++q) {
        m.to_physical(rule.xi[q], rule.eta[q], x[e * Q + q], y[e * Q + q]);
        if (w)
          w[e * Q + q] = rule.w[q] * jac;
      }
    }
  }

  void project(int rule_order, const double *values) override {
    const Rule2D rule = triangle_rule(rule_order);
    const int Q = rule.size();
    std::vector<double> c(static_cast<std::size_t>(M_) * ne_, 0.0);
    for (int q = 0; q < Q; ++q) {
      const auto b = dubiner(rule.xi[q], rule.eta[q], p_);
      for (std::int64_t e = 0; e < ne_; ++e)
        for (int m = 0; m < M_; ++m)
          c[static_cast<std::int64_t>(m) * ne_ + e] += rule.w[q] * values[e * Q + q] * b[m];
    }
    set_state(c.data());
  }

  void evaluate(int rule_order, double *values) override {
    const Rule2D rule = triangle_rule(rule_order);
    const int Q = rule.size();
    std::vector<double> c(static_cast<std::size_t>(M_) * ne_);
    get_state(c.data());
    std::vector<std::vector<double>> basis(Q);
    for (int q = 0; q < Q; ++q)
      basis[q] = dubiner(rule.xi[q], rule.eta[q], p_);
    for (std::int64_t e = 0; e < ne_; ++e)
      for (int q = 0; q < Q; ++q) {
        double s = 0.0;
        for (int m = 0; m < M_; ++m)
          s += c[static_cast<std::int64_t>(m) * ne_ + e] * basis[q][m];
        values[e * Q + q] = s;
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

  // triangle_scalar_cfl_timestep: fixed by the mesh and the velocity.
  double stable_dt(double cfl) override {
    const double speed = std::hypot(cfg_.velocity_x, cfg_.velocity_y);
    if (ne_ == 0 || speed == 0.0)
      return 0.0;
    return cfl * length_ / (speed * (2.0 * p_ + 1.0));
  }

  void step(double dt) override {
    enqueue_step(dt);
    cuda_check(cudaGetLastError(), "stage launch");
  }

  void limit() override {}

  void advance(double cfl, std::int64_t steps) override {
    const double dt = stable_dt(cfl);
    for (std::int64_t n = 0; n < steps; ++n)
      enqueue_step(dt);
    cuda_check(cudaGetLastError(), "advance");
  }

  void flags(std::uint8_t *out) override {
    cuda_check(cudaMemcpyAsync(out, d_flags_.get(), 3 * ne_, cudaMemcpyDeviceToHost, stream_),
               "flags");
    cuda_check(cudaStreamSynchronize(stream_), "flags");
  }

  // scalar_diagnostics.cpp:29-36 (energy = mass).
  void mass_energy(double &mass, double &energy) override {
    std::vector<double> c0(ne_);
    cuda_check(cudaMemcpyAsync(c0.data(), d_u_.get(), ne_ * sizeof(double), cudaMemcpyDeviceToHost,
                               stream_),
               "mass");
    cuda_check(cudaStreamSynchronize(stream_), "mass");
    mass = 0.0;
    for (std::int64_t e = 0; e < ne_; ++e)
      mass += std::sqrt(2.0) * mesh_.maps[e].jacobian_determinant() * c0[e];
    energy = mass;
  }

private:
  void enqueue_step(double dt) {
    StageArgs a;
    a.mesh.ne = ne_;
    a.mesh.geo = d_geo_.get();
    a.mesh.slot_nbr = d_slot_nbr_.get();
    a.mesh.slot_code = d_slot_code_.get();
    a.mesh.slot_geo = d_slot_geo_.get();
    a.mesh.donor = d_donor_.get();
    a.mesh.donor_basis = d_donor_basis_.get();
    a.face_table = d_face_table_.get();
    a.dt = nullptr;
    a.dt_value = dt;
    a.velocity_x = cfg_.velocity_x;
    a.velocity_y = cfg_.velocity_y;
    double *ins[3] = {d_u_.get(), d_e_.get(), d_s_.get()};
    double *outs[3] = {d_e_.get(), d_s_.get(), d_u_.get()};
    for (int k = 0; k < 3; ++k) {
      a.stage = k;
      a.in = ins[k];
      a.u0 = d_u_.get();
      a.out = outs[k];
      stage_begin();
      launch_scalar_tri_stage_f64(p_, a, stream_);
      stage_end();
      count_launches(1);
    }
  }

  wasl_gpu_config cfg_;
  TriTopology mesh_;
  int p_, M_;
  std::int64_t ne_ = 0;
  double length_ = 0.0;
  DeviceArray<double> d_geo_, d_slot_geo_, d_donor_basis_, d_u_, d_e_, d_s_;
  DeviceArray<std::int32_t> d_slot_nbr_, d_donor_;
  DeviceArray<std::uint8_t> d_slot_code_, d_flags_;
  DeviceArray<unsigned char> d_face_table_;
};

std::unique_ptr<Solver> make_scalar_tri_solver(const wasl_gpu_config &cfg, TriTopology &&topo,
                                               const PartBoundary *part) {
  return std::make_unique<ScalarTriSolver>(cfg, std::move(topo), part);
}

} // namespace wasl_b200
