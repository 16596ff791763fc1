// Host-side mesh setup: canonical topology and the per-mesh data the kernels read.
//
// The topology follows the reference's canonical rules so face indices, and with
// them the flux summation order, are the same:
//   * triangles reoriented counter-clockwise (build_triangle_mesh.cpp:38-65);
//   * an edge's left element is the first element (by index, then local edge)
//     that has it, the right element the second; faces sorted by
//     (left element, left local edge) (build_triangle_mesh.cpp:67-148);
//   * the stored normal is the left element's outward unit normal.
// Lines are oriented left to right, stably sorted by left end, with faces
// [left boundary, interior pairs..., right boundary] (build_line_mesh.cpp:14-84).
#pragma once

#include <cstdint>
#include <string>

#include "element_grid.hpp"
#include <vector>

namespace wasl_b200 {

struct TriMap {
  double x0, y0, x1, y1, x2, y2;

  double ax() const { return x1 - x0; }
  double ay() const { return y1 - y0; }
  double bx() const { return x2 - x0; }
  double by() const { return y2 - y0; }
  double det_a() const { return ax() * by() - bx() * ay(); }
  double jacobian_determinant() const { return det_a() / 4.0; }
  int orientation() const { return det_a() > 0.0 ? 1 : -1; }
  void to_physical(double xi, double eta, double &x, double &y) const;
  void to_reference(double x, double y, double &xi, double &eta) const;
  void edge_vector(int edge, double &ex, double &ey) const;
  double edge_length(int edge) const;
  void edge_normal(int edge, double &nx, double &ny) const;
  void shift(double ox, double oy);
};

struct TriTopology {
  std::int64_t element_count = 0;
  std::vector<TriMap> maps;               // [element], counter-clockwise
  std::vector<std::int64_t> nodes;        // [element][3] node tags after reorientation
  std::vector<std::int32_t> face_left;    // [face]
  std::vector<std::int32_t> face_right;   // [face], -1 on a boundary
  std::vector<std::int32_t> face_left_edge, face_right_edge;
  std::vector<std::uint8_t> face_flip;    // the two sides traverse the edge oppositely
  std::vector<double> face_nx, face_ny;   // left element's outward unit normal
  std::vector<double> face_scale;         // physical / reference length of the left edge
  std::int64_t face_count() const { return static_cast<std::int64_t>(face_left.size()); }
};

// Throws std::runtime_error with the reference's messages on a bad mesh.
TriTopology build_triangle_topology(std::int64_t node_count, const std::int64_t *node_tags,
                                    const double *node_xy, std::int64_t element_count,
                                    const std::int64_t *element_nodes);

struct LineTopology {
  std::int64_t element_count = 0;
  std::vector<double> x_left, x_right;
  std::vector<std::int32_t> face_left, face_right; // right -1 on a boundary
  std::vector<double> face_normal;
  std::int64_t face_count() const { return static_cast<std::int64_t>(face_left.size()); }
};

LineTopology build_line_topology(std::int64_t node_count, const std::int64_t *node_tags,
                                 const double *node_x, std::int64_t element_count,
                                 const std::int64_t *element_nodes);

// Periodic images of every boundary edge point, located once
// (cpp/src/boundaries/periodic_triangle_trace.cpp:40-67).  The donor of each
// point is the first element, by index, whose reference coordinates contain it
// within 1e-10; a uniform bucket grid narrows the candidates, so the search is
// near-linear instead of the reference's O(boundary x elements), with the same
// answer.  Indexed by boundary face b (the faces without a right element, in
// ascending face index): donors [b][point], basis [b][point][mode].
struct PeriodicTrace {
  std::vector<std::int32_t> donors;
  std::vector<double> basis;
};
PeriodicTrace periodic_trace(const TriTopology &mesh, int p);

// The boundary of one part of a partitioned periodic mesh, given by the
// caller instead of found by the donor search: per boundary face b of the
// part's mesh (ascending face index) and edge point q, the donor element
// (an index into the part's elements) and the donor's basis at the point's
// periodic image, donors [b][q], basis [b][q][mode]; donor -1 on every point
// of a face marks a face where the part's ghost region ends, whose exterior
// is its own element's trace.
struct PartBoundary {
  std::int64_t faces = 0;
  const std::int32_t *donors = nullptr;
  const double *basis = nullptr;
};

// The periodic trace of a part (owner faces filled with the owner and its
// own basis at its edge points); stencil_donors: the donors with -1 kept on
// owner faces, for triangle_stencil.  Throws std::invalid_argument when the
// boundary does not fit the mesh.
PeriodicTrace part_trace(const TriTopology &mesh, int p, const PartBoundary &part,
                         std::vector<std::int32_t> &stencil_donors);

// The mesh's bounding box.
struct Box {
  double min_x, max_x, min_y, max_y;
};
Box bounding_box(const TriTopology &mesh);

// The boundary edge points' periodic images, in boundary face order: point
// [b][q] of boundary face b is its left element's edge point q moved by one
// period across the box (the face's normal is axis-aligned; otherwise throws
// the reference's "2D periodic boundaries require an axis-aligned box").
struct PeriodicImages {
  std::int64_t faces = 0;  // boundary faces with images (all, unless misaligned)
  int points = 0;          // per face
  bool misaligned = false; // a boundary face after the last one here is not axis-aligned
  std::vector<double> x, y;
};
PeriodicImages periodic_images(const TriTopology &mesh, int p);

// The donor search's grid over this mesh (element_grid.hpp).
GridShape element_grid_shape(const TriTopology &mesh);

// The cells holding image points, ascending, each with its points (indices
// into PeriodicImages::x/y): point[start[r] .. start[r + 1]) lie in cells[r].
struct ImageCells {
  std::vector<int> cells;
  std::vector<std::int64_t> start, point;
};
ImageCells image_cells(const GridShape &g, const PeriodicImages &images);

// The periodic trace from each image's donor (-1: none found, which throws
// the reference's "periodic 2D trace has no donor element"): donors as given,
// basis evaluated in the donor's reference coordinates.
PeriodicTrace periodic_trace_from_donors(const TriTopology &mesh, int p,
                                         const PeriodicImages &images,
                                         std::vector<std::int32_t> &&donors);

// The face slots and boundary lists the triangle stage kernels read, built in
// ascending global face index (the reference's flux summation order):
//   geo [5][ne]: ax, ay, bx, by (the affine map's columns), 1/det(J);
//   slot_nbr/slot_code/slot_face [3][ne], slot_geo [3][3][ne] (normal x, y,
//   edge scale); code bit 0: this element is the face's left side, bits 1-2
//   left local edge, bits 3-4 right local edge, bit 5 orientation flip;
//   face_right [face]: the right element, or -(b+1) for boundary face b;
//   boundary lists in boundary order, with each boundary face's periodic
//   donors [b][QF] and donor basis [b][QF][M] when a trace is given.
struct TriSlots {
  std::vector<double> geo;
  std::vector<std::int32_t> slot_nbr, slot_face;
  std::vector<std::uint8_t> slot_code;
  std::vector<double> slot_geo;
  std::vector<std::int32_t> face_right, left_slot;
  std::vector<std::uint8_t> face_code;
  std::vector<double> face_normal;        // [2][face]
  std::vector<std::int32_t> bnd_element;
  std::vector<std::uint8_t> bnd_edge;
  std::vector<double> bnd_normal;         // [2][boundary]
  std::vector<std::int32_t> donors;
  std::vector<double> donor_basis;
  std::int64_t boundary_count = 0;
};
TriSlots build_tri_slots(const TriTopology &mesh, const PeriodicTrace *trace, int QF, int M);

// Immediate-neighbour limiter stencil (cpp/include/wasl/limiting/euler_limiter_stencil.hpp:19-50).
struct LimiterStencil {
  int mode_count = 0;
  int maximum_neighbors = 0;
  int highest_degree_begin = 0;
  std::vector<std::int32_t> neighbors; // [element][candidate], -1 if absent
  std::vector<double> transforms;      // [element][candidate][target][source]
  std::vector<double> normal_x, normal_y;
  std::vector<double> check_basis;     // [point][mode]
  int check_point_count() const {
    return mode_count ? static_cast<int>(check_basis.size()) / mode_count : 0;
  }
};

// periodic_donors may be empty (open boundaries).
// periodic_donors: PeriodicTrace::donors (empty without periodic faces).
// Without `transforms` the candidate transforms are left empty (the device
// builds them, setup_device.cu).
LimiterStencil triangle_stencil(const TriTopology &mesh, int p,
                                const std::vector<std::int32_t> &periodic_donors,
                                bool transforms = true);

// The period a neighbour's copy is shifted by in the limiter stencil: one
// period toward the target when their centroids lie more than half a period
// apart (euler_limiter_stencil_triangle.cpp:51-79).
WASL_HD double period_shift(double gap, double period) {
  return gap > 0.5 * period ? period : gap < -0.5 * period ? -period : 0.0;
}
LimiterStencil line_stencil(const LineTopology &mesh, int p, bool periodic);

// cpp/src/time/cfl_timestep.cpp:14-30
double minimum_altitude(const TriTopology &mesh);
double minimum_length(const LineTopology &mesh);

} // namespace wasl_b200
