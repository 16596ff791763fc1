// Host-side setup shared by the single-case and batched triangle solvers:
// periodic face pairing and the tile kernel's element-centric slots, and
// quadrature, L2 projection and evaluation on a triangle mesh.
#pragma once

#include <cstdint>
#include <vector>

#include "mesh.hpp"

namespace wasl_b200 {

// The mixed form evaluates each periodic face pair once, as one face between
// the two elements: the lower-numbered face of the pair is kept (its element
// is the left side, the donor the right), the other is marked skipped
// (face_code bit 7) and its element's slot is re-pointed to the kept face
// (slot_code bit 6: its basis on the face is the donor basis row), with the
// kept face's normal and scale.  Needs every boundary face to have one donor
// whose boundary face points back; returns false (slots untouched) otherwise.
// A face whose donor is its own element (a partition part's cut face, which
// takes its own trace) stays unpaired, and the tile and patch arrays below
// give it the transmissive exterior.
// basis32: the donor basis [boundary face][QF][M] in FP32.
bool pair_periodic_faces(const TriTopology &mesh, int QF, TriSlots &t, std::vector<float> &basis32);

// Element-centric slots of the tile kernel (kernels.hpp TileSlots) from the
// face slots after pairing; boundary is WASL_TRANSMISSIVE or WASL_PERIODIC
// (paired).
struct TileSlotArrays {
  std::vector<std::int32_t> nbr, aux;
  std::vector<std::uint8_t> code;
};
TileSlotArrays build_tile_slots(const TriTopology &mesh, const TriSlots &t, int boundary, int QF);

// Per-element, per-local-edge arrays of the patch kernel, [3][ne] (the
// element's local edges 0..2, not its faces in face order):
//   nbr   the element across the edge; -1 on a transmissive boundary.  A
//         periodic face pair is one face between the two elements (the
//         lower-numbered face of the pair is kept: its element is the left
//         side, with that face's normal and scale).
//   info  bit 0: this element is the face's left side (on a boundary: set);
//         bits 1-2: the neighbour's local edge; bit 3: the neighbour's edge
//         points run in the opposite order (its point QF-1-q is this face's
//         point q).
//   geo   [3 edges][3][ne]: the face's normal (left to right) and scale.
// The point order of every face is matched on physical coordinates (periodic
// pairs relative to each edge's midpoint); returns false, leaving `out`
// incomplete, where a face's points do not match (a non-conforming mesh) or a
// periodic boundary face has no single partner.
struct PatchEdgeArrays {
  std::vector<std::int32_t> nbr;
  std::vector<std::uint8_t> info;
  std::vector<double> geo;
};
bool build_patch_edges(const TriTopology &mesh, const TriSlots &t, int boundary, int QF,
                       PatchEdgeArrays &out);

// An element order along a space-filling (Morton) curve of the element
// centroids: order[i] is the element stored at position i.  Consecutive
// positions are then close in space, so a patch of consecutive elements
// shares most of its faces.  Ties keep the mesh order.
std::vector<std::int32_t> morton_order(const TriTopology &mesh);

// Physical points and weights (reference weight x |det J|) of the collapsed
// rule of order r on every element, packed [element][point]; w may be null.
void tri_quadrature(const TriTopology &mesh, int rule_order, double *x, double *y, double *w);

// L2 projection of point values [element][point][variable] at that rule's
// points onto P_p: coefficients [variable][mode][element]
// (cpp/include/wasl/dg/l2_projection.hpp:57-76).
std::vector<double> tri_project(const TriTopology &mesh, int p, int variables, int rule_order,
                                const double *values);

// Coefficients [variable][mode][element] evaluated at the rule's points,
// [element][point][variable].
void tri_evaluate(const TriTopology &mesh, int p, int variables, int rule_order,
                  const double *coefficients, double *values);

} // namespace wasl_b200
