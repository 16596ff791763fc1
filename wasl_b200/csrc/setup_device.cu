// Mesh setup on the device (setup_device.hpp).  Compiled with --fmad=false:
// every product and sum rounds as the host setup's (mesh.cpp, built with
// -ffp-contract=off), so the results are the host's bit for bit.
#include "setup_device.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <stdexcept>

#include "basis.hpp"
#include "element_grid.hpp"
#include "exact_power.hpp"
#include "parallel.hpp"

namespace wasl_b200 {
namespace {

constexpr int kMaxRule = 16, kMaxModes = 10; // the order-p collapsed rule and modes, p <= 3

// The stencil's reference tables (triangle_stencil, mesh.cpp): the target
// rule's points, weights and basis, and each mode's (i, j) and norm.
struct StencilTables {
  double xi[kMaxRule], eta[kMaxRule], w[kMaxRule];
  double tb[kMaxRule * kMaxModes]; // [point][mode]
  double norm[kMaxModes];
  int mode_i[kMaxModes], mode_j[kMaxModes];
};
__constant__ StencilTables c_stencil;

// jacobi() of basis.hpp, expression for expression.
__device__ __forceinline__ double device_jacobi(double x, int n, double alpha, double beta) {
  if (n <= 0)
    return 1.0;
  double prev = 1.0;
  double curr = 0.5 * (alpha - beta + (alpha + beta + 2.0) * x);
  for (int k = 1; k < n; ++k) {
    const double ab = 2.0 * k + alpha + beta;
    const double a = 2.0 * (k + 1) * (k + alpha + beta + 1.0) * ab;
    const double b = (ab + 1.0) * (ab * (ab + 2.0) * x + (alpha * alpha - beta * beta));
    const double c = 2.0 * (k + alpha) * (k + beta) * (ab + 2.0);
    const double next = (b * curr - c * prev) / a;
    prev = curr;
    curr = next;
  }
  return curr;
}

__device__ __forceinline__ double device_collapsed(double xi, double eta) {
  return (eta < 1.0) ? (2.0 + 2.0 * xi) / (1.0 - eta) - 1.0 : -1.0;
}

// Rule point q of target element e in the reference coordinates of its
// neighbour nb, the neighbour moved by a period when their centroids lie
// more than half a period apart: triangle_stencil's TriMap arithmetic.
__device__ __forceinline__ void source_point(const double *__restrict__ maps, std::int64_t e,
                                             std::int64_t nb, int q, double width, double height,
                                             double &xi, double &eta) {
  const double *t = maps + 6 * e;
  double v[6];
#pragma unroll
  for (int r = 0; r < 6; ++r)
    v[r] = maps[6 * nb + r];
  const double ox = period_shift((t[0] + t[2] + t[4] - v[0] - v[2] - v[4]) / 3.0, width);
  const double oy = period_shift((t[1] + t[3] + t[5] - v[1] - v[3] - v[5]) / 3.0, height);
  v[0] += ox, v[2] += ox, v[4] += ox;
  v[1] += oy, v[3] += oy, v[5] += oy;
  const double rx = c_stencil.xi[q], ry = c_stencil.eta[q];
  const double x = t[0] + 0.5 * ((t[2] - t[0]) * (rx + 1.0) + (t[4] - t[0]) * (ry + 1.0));
  const double y = t[1] + 0.5 * ((t[3] - t[1]) * (rx + 1.0) + (t[5] - t[1]) * (ry + 1.0));
  grid_to_reference(v, x, y, xi, eta);
}

// Pass 1, one thread per (element, candidate, rule point) of the chunk: the
// powers ((1 - eta) / 2)^i, i = 2..P, rounded, into warp[i - 2][entry]; the
// unsettled ones listed (entry * 4 + i, base) for the host's pow.
template <int P>
__global__ void stencil_powers(const double *__restrict__ maps, const std::int32_t *__restrict__ nbrs,
                               const std::int32_t *__restrict__ order, std::int64_t first,
                               std::int64_t entries, double width, double height,
                               double *__restrict__ warp, unsigned *__restrict__ unsettled,
                               unsigned *__restrict__ codes, double *__restrict__ bases) {
  constexpr int Q = (P + 1) * (P + 1);
  const std::int64_t idx = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= entries)
    return;
  const std::int64_t s = first + idx / (3 * Q);
  const int k = static_cast<int>((idx / Q) % 3), q = static_cast<int>(idx % Q);
  const std::int64_t e = order ? order[s] : s;
  const std::int32_t nb = nbrs[3 * e + k];
  if (nb < 0)
    return;
  double xi, eta;
  source_point(maps, e, nb, q, width, height, xi, eta);
  const double half = 0.5 * (1.0 - eta);
  bool open = false;
  warp[idx] = power2(half, &open);
  if (open) {
    const unsigned at = atomicAdd(unsettled, 1u);
    codes[at] = static_cast<unsigned>(idx) * 4u + 2u;
    bases[at] = half;
  }
  if constexpr (P >= 3) {
    warp[entries + idx] = power3(half, &open);
    if (open) {
      const unsigned at = atomicAdd(unsettled, 1u);
      codes[at] = static_cast<unsigned>(idx) * 4u + 3u;
      bases[at] = half;
    }
  }
}

// The host's powers written over the unsettled entries.
__global__ void patch_powers(unsigned count, const unsigned *__restrict__ codes,
                             const double *__restrict__ values, std::int64_t entries,
                             double *__restrict__ warp) {
  const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count)
    return;
  const unsigned code = codes[k];
  warp[static_cast<std::int64_t>((code & 3u) - 2u) * entries + (code >> 2)] = values[k];
}

// Pass 2, one thread per (element, candidate, source mode) of the chunk: the
// transform's column for that source mode, transform[t][sm] = sum over the
// rule points of w_q (modal sum of the unit vector e_sm at the point)
// phi_t(point), accumulated in point order as the host does.  The modal sum
// of a unit vector is 0.0 + phi_sm (adding the zero products leaves a
// nonzero value unchanged and turns -0.0 into +0.0).
template <int P>
__global__ void stencil_columns(const double *__restrict__ maps, const std::int32_t *__restrict__ nbrs,
                                const std::int32_t *__restrict__ order, std::int64_t first,
                                std::int64_t elements, double width, double height,
                                const double *__restrict__ warp, std::int64_t entries,
                                double *__restrict__ out) {
  constexpr int Q = (P + 1) * (P + 1), M = (P + 1) * (P + 2) / 2;
  const std::int64_t idx = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= elements * 3 * M)
    return;
  const std::int64_t local = idx / (3 * M), s = first + local;
  const int k = static_cast<int>((idx / M) % 3), sm = static_cast<int>(idx % M);
  const std::int64_t e = order ? order[s] : s;
  const std::int32_t nb = nbrs[3 * e + k];
  double *matrix = out + (3 * s + k) * M * M;
  if (nb < 0) {
#pragma unroll
    for (int t = 0; t < M; ++t)
      matrix[t * M + sm] = 0.0;
    return;
  }
  const int i = c_stencil.mode_i[sm], j = c_stencil.mode_j[sm];
  const double norm = c_stencil.norm[sm];
  double acc[M];
#pragma unroll
  for (int t = 0; t < M; ++t)
    acc[t] = 0.0;
  for (int q = 0; q < Q; ++q) {
    double xi, eta;
    source_point(maps, e, nb, q, width, height, xi, eta);
    const double a = device_collapsed(xi, eta);
    const double half = 0.5 * (1.0 - eta);
    const double pi = device_jacobi(a, i, 0.0, 0.0);
    const double power =
        i == 0 ? 1.0 : i == 1 ? half : warp[(i - 2) * entries + (local * 3 + k) * Q + q];
    const double qj = device_jacobi(eta, j, 2.0 * i + 1.0, 0.0);
    const double value = 0.0 + norm * pi * power * qj;
#pragma unroll
    for (int t = 0; t < M; ++t)
      acc[t] += c_stencil.w[q] * value * c_stencil.tb[q * M + t];
  }
#pragma unroll
  for (int t = 0; t < M; ++t)
    matrix[t * M + sm] = acc[t];
}

__global__ void fill_int(std::int32_t *p, std::int64_t n, std::int32_t value) {
  const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n)
    p[i] = value;
}

// One thread per element: the smallest element containing each image point
// among the elements whose padded box covers the point's cell.
__global__ void donor_sweep(const double *__restrict__ maps, std::int64_t elements, GridShape g,
                            const int *__restrict__ cells, int cell_count,
                            const std::int64_t *__restrict__ start,
                            const std::int64_t *__restrict__ point, const double *__restrict__ px,
                            const double *__restrict__ py, std::int32_t *__restrict__ best) {
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= elements)
    return;
  double v[6];
#pragma unroll
  for (int r = 0; r < 6; ++r)
    v[r] = maps[6 * e + r];
  int i0, i1, j0, j1;
  grid_cell_range(g, v, i0, i1, j0, j1);
  for (int j = j0; j <= j1; ++j)
    for (int i = i0; i <= i1; ++i) {
      const int c = j * g.nx + i;
      int lo = 0, hi = cell_count; // first cell >= c
      while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (cells[mid] < c)
          lo = mid + 1;
        else
          hi = mid;
      }
      if (lo == cell_count || cells[lo] != c)
        continue;
      for (std::int64_t k = start[lo]; k < start[lo + 1]; ++k) {
        const std::int64_t pt = point[k];
        double xi, eta;
        grid_to_reference(v, px[pt], py[pt], xi, eta);
        if (grid_contains(xi, eta))
          atomicMin(best + pt, static_cast<std::int32_t>(e));
      }
    }
}

unsigned blocks_for(std::int64_t n, int threads) {
  return static_cast<unsigned>((n + threads - 1) / threads);
}

template <typename T> void copy_in(DeviceArray<T> &d, const std::vector<T> &h, cudaStream_t s) {
  d.upload(h, s);
}

template <int P>
void transforms_for(const TriTopology &mesh, const std::vector<std::int32_t> &neighbors,
                    const std::vector<std::int32_t> &order, const double *d_maps,
                    double *d_transforms, cudaStream_t s) {
  constexpr int Q = (P + 1) * (P + 1), M = (P + 1) * (P + 2) / 2;
  static_assert(Q <= kMaxRule && M <= kMaxModes, "stencil tables too small");
  const std::int64_t ne = mesh.element_count;
  StencilTables tables{};
  const Rule2D rule = triangle_rule(P);
  for (int q = 0; q < Q; ++q) {
    tables.xi[q] = rule.xi[q];
    tables.eta[q] = rule.eta[q];
    tables.w[q] = rule.w[q];
    const auto b = dubiner(rule.xi[q], rule.eta[q], P);
    for (int t = 0; t < M; ++t)
      tables.tb[q * M + t] = b[t];
  }
  for (int n = 0, m = 0; n <= P; ++n)
    for (int i = 0; i <= n; ++i, ++m) {
      tables.mode_i[m] = i;
      tables.mode_j[m] = n - i;
      tables.norm[m] = dubiner_norm(i, n);
    }
  cuda_check(cudaMemcpyToSymbolAsync(c_stencil, &tables, sizeof tables, 0,
                                     cudaMemcpyHostToDevice, s),
             "stencil tables");
  const Box box = bounding_box(mesh);
  const double width = box.max_x - box.min_x, height = box.max_y - box.min_y;

  DeviceArray<std::int32_t> d_nbrs, d_order;
  copy_in(d_nbrs, neighbors, s);
  if (!order.empty())
    copy_in(d_order, order, s);
  const std::int32_t *ord = order.empty() ? nullptr : d_order.get();

  // Chunks of at most 2^24 (element, candidate, point) entries.
  const std::int64_t chunk = std::max<std::int64_t>(1, (std::int64_t{1} << 24) / (3 * Q));
  const std::int64_t most = std::min(ne, chunk) * 3 * Q;
  DeviceArray<double> warp, bases, values;
  DeviceArray<unsigned> codes, unsettled;
  std::vector<unsigned> h_codes;
  std::vector<double> h_bases, h_values;
  if (P >= 2) {
    warp.resize(static_cast<std::size_t>(most) * (P - 1));
    codes.resize(static_cast<std::size_t>(most) * (P - 1));
    bases.resize(static_cast<std::size_t>(most) * (P - 1));
    values.resize(static_cast<std::size_t>(most) * (P - 1));
    unsettled.resize(1);
  }
  for (std::int64_t first = 0; first < ne; first += chunk) {
    const std::int64_t elements = std::min(chunk, ne - first), entries = elements * 3 * Q;
    if (P >= 2) {
      cuda_check(cudaMemsetAsync(unsettled.get(), 0, sizeof(unsigned), s), "memset");
      stencil_powers<P><<<blocks_for(entries, 256), 256, 0, s>>>(
          d_maps, d_nbrs.get(), ord, first, entries, width, height, warp.get(), unsettled.get(),
          codes.get(), bases.get());
      unsigned count = 0;
      cuda_check(cudaMemcpyAsync(&count, unsettled.get(), sizeof count, cudaMemcpyDeviceToHost, s),
                 "unsettled count");
      cuda_check(cudaStreamSynchronize(s), "stencil powers");
      if (count > 0) {
        h_codes.resize(count);
        h_bases.resize(count);
        h_values.resize(count);
        cuda_check(cudaMemcpyAsync(h_codes.data(), codes.get(), count * sizeof(unsigned),
                                   cudaMemcpyDeviceToHost, s),
                   "unsettled codes");
        cuda_check(cudaMemcpyAsync(h_bases.data(), bases.get(), count * sizeof(double),
                                   cudaMemcpyDeviceToHost, s),
                   "unsettled bases");
        cuda_check(cudaStreamSynchronize(s), "unsettled powers");
        parallel_for(count, [&](std::int64_t begin, std::int64_t end) {
          for (std::int64_t k = begin; k < end; ++k)
            h_values[k] = std::pow(h_bases[k], static_cast<double>(h_codes[k] & 3u));
        });
        cuda_check(cudaMemcpyAsync(values.get(), h_values.data(), count * sizeof(double),
                                   cudaMemcpyHostToDevice, s),
                   "library powers");
        patch_powers<<<blocks_for(count, 256), 256, 0, s>>>(count, codes.get(), values.get(),
                                                            entries, warp.get());
      }
    }
    stencil_columns<P><<<blocks_for(elements * 3 * M, 128), 128, 0, s>>>(
        d_maps, d_nbrs.get(), ord, first, elements, width, height, warp.get(), entries,
        d_transforms);
    cuda_check(cudaGetLastError(), "stencil transforms");
    // The host buffers above are reused by the next chunk.
    cuda_check(cudaStreamSynchronize(s), "stencil transforms");
  }
}

} // namespace

void upload_maps(const TriTopology &mesh, DeviceArray<double> &maps, cudaStream_t s) {
  static_assert(sizeof(TriMap) == 6 * sizeof(double), "TriMap is six doubles");
  maps.resize(static_cast<std::size_t>(6) * mesh.element_count);
  cuda_check(cudaMemcpyAsync(maps.get(), mesh.maps.data(), maps.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s),
             "upload maps");
}

PeriodicTrace periodic_trace_device(const TriTopology &mesh, int p, const double *d_maps,
                                    cudaStream_t s) {
  const PeriodicImages images = periodic_images(mesh, p);
  const std::int64_t n = static_cast<std::int64_t>(images.x.size());
  std::vector<std::int32_t> donors(n, -1);
  if (n > 0) {
    const GridShape g = element_grid_shape(mesh);
    const ImageCells ic = image_cells(g, images);
    DeviceArray<int> cells;
    DeviceArray<std::int64_t> start, point;
    DeviceArray<double> px, py;
    DeviceArray<std::int32_t> best(n);
    copy_in(cells, ic.cells, s);
    copy_in(start, ic.start, s);
    copy_in(point, ic.point, s);
    copy_in(px, images.x, s);
    copy_in(py, images.y, s);
    fill_int<<<blocks_for(n, 256), 256, 0, s>>>(best.get(), n, INT_MAX);
    donor_sweep<<<blocks_for(mesh.element_count, 256), 256, 0, s>>>(
        d_maps, mesh.element_count, g, cells.get(), static_cast<int>(ic.cells.size()),
        start.get(), point.get(), px.get(), py.get(), best.get());
    cuda_check(cudaGetLastError(), "donor sweep");
    cuda_check(cudaMemcpyAsync(donors.data(), best.get(), n * sizeof(std::int32_t),
                               cudaMemcpyDeviceToHost, s),
               "donors");
    cuda_check(cudaStreamSynchronize(s), "donor sweep");
    for (auto &d : donors)
      if (d == INT_MAX)
        d = -1;
  }
  return periodic_trace_from_donors(mesh, p, images, std::move(donors));
}

void stencil_transforms_device(const TriTopology &mesh, int p,
                               const std::vector<std::int32_t> &neighbors,
                               const std::vector<std::int32_t> &order, const double *d_maps,
                               double *d_transforms, cudaStream_t s) {
  switch (p) {
  case 1: transforms_for<1>(mesh, neighbors, order, d_maps, d_transforms, s); break;
  case 2: transforms_for<2>(mesh, neighbors, order, d_maps, d_transforms, s); break;
  case 3: transforms_for<3>(mesh, neighbors, order, d_maps, d_transforms, s); break;
  default: throw std::invalid_argument("stencil transforms on the device: order 1..3");
  }
}

} // namespace wasl_b200
