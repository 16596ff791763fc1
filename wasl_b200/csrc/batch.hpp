// The batched 2D Euler solver behind wasl_batch_* (see batch_solver.cu).
#pragma once

#include <array>
#include <atomic>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "autotune.hpp"
#include "kernels.hpp"
#include "mesh.hpp"
#include "solver.hpp"

namespace wasl_b200 {

class BatchSolver {
public:
  BatchSolver(const wasl_batch_config &cfg, std::int64_t case_count, const int *orders,
              const std::int64_t *node_counts, const std::int64_t *node_tags,
              const double *node_xy, const std::int64_t *element_counts,
              const std::int64_t *element_nodes);
  ~BatchSolver();
  BatchSolver(const BatchSolver &) = delete;
  BatchSolver &operator=(const BatchSolver &) = delete;

  std::int64_t cases() const { return cases_; }
  std::int64_t case_elements(std::int64_t c) const;
  int case_modes(std::int64_t c) const;
  std::int64_t total_elements() const { return total_elements_; }
  std::int64_t total_dof() const { return total_dof_; }
  void set_state(std::int64_t c, const double *host);
  void get_state(std::int64_t c, double *host);
  void quadrature(std::int64_t c, int rule, double *x, double *y, double *w) const;
  void project(std::int64_t c, int rule, const double *values);
  void advance(double cfl, std::int64_t steps);
  void limit();
  void times(double *time, double *dt);
  void status(int *out);
  int tuning(int p, double *ms, int capacity, int &count) const;
  cudaStream_t stream() const { return stream_; }
  std::int64_t launches_per_step() const { return launches_per_step_; }
  std::int64_t launches() const { return launches_; }
  bool graph() const { return graph_exec_ != nullptr; }

private:
  struct Group {
    Group();
    ~Group();
    int p = 0, M = 0, rule = 0;
    std::int64_t ne = 0;
    std::vector<std::int64_t> cases;
    int shape = 0;
    TuneResult tuning;
    int highest_degree_begin = 0, check_points = 0;
    DeviceArray<double> u, e, s, geo, slot_geo, transforms, normal_x, normal_y, check, limited,
        basis64, check_bound;
    DeviceArray<std::int32_t> tile_nbr, tile_aux, neighbors, troubled, count, element_case, rough;
    DeviceArray<std::uint8_t> tile_code, flags;
    DeviceArray<float> basis32;
    DeviceArray<unsigned char> face_table, face_table64;
    std::array<DeviceArray<TileWork>, kTileShapeCount> work;
    std::array<std::int64_t, kTileShapeCount> work_count{};
  };

  void check_case(std::int64_t c) const;
  void copy_case(std::int64_t c, double *host, bool to_device);
  StageArgs stage_args(const Group &g, int stage) const;
  LimitArgs limit_args(const Group &g, double *state) const;
  void tune();
  void enqueue_step(double cfl);
  void check_error();

  wasl_batch_config cfg_;
  std::int64_t cases_ = 0;
  cudaStream_t stream_ = nullptr;
  std::vector<std::unique_ptr<Group>> groups_;
  std::vector<int> case_group_;
  std::vector<std::int64_t> case_offset_;
  std::vector<TriTopology> meshes_; // maps only, for quadrature and projection
  std::int64_t total_elements_ = 0, total_dof_ = 0;
  DeviceArray<double> d_length_, d_dt_, d_time_;
  DeviceArray<int> d_p_, d_status_;
  DeviceArray<unsigned long long> d_speed_, d_error_;
  bool tuned_ = false;
  cudaGraphExec_t graph_exec_ = nullptr;
  double graph_cfl_ = 0.0;
  std::int64_t launches_per_step_ = 0, launches_ = 0;
};

} // namespace wasl_b200
