// Mesh setup on the device: the periodic donor search and the limiter
// stencil's candidate transforms, the two setup steps whose work grows with
// the element count times the basis size.  Both give the host setup's
// results bit for bit (mesh.cpp: periodic_trace, triangle_stencil).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "mesh.hpp"
#include "solver.hpp"

namespace wasl_b200 {

// The element maps [element][6] (x0, y0, x1, y1, x2, y2) in the caller's
// order, on the device.
void upload_maps(const TriTopology &mesh, DeviceArray<double> &maps, cudaStream_t s);

// periodic_trace (mesh.cpp) with the element sweep on the device: the host
// places the periodic images and bins them into the grid's cells; one thread
// per element tests the images in the cells its padded box covers and keeps
// the smallest containing element per image (atomicMin); the host then
// evaluates the basis at each image in its donor.
PeriodicTrace periodic_trace_device(const TriTopology &mesh, int p, const double *d_maps,
                                    cudaStream_t s);

// The limiter stencil's candidate transforms (triangle_stencil's
// `transforms`, mesh.cpp) built on the device into d_transforms
// [storage element][candidate][target][source]: storage element i is the
// caller's element order[i] (identity when order is empty).  neighbors:
// LimiterStencil::neighbors, [caller element][3] caller ids.
//
// The source basis takes ((1 - eta) / 2)^i with the C library's pow; the
// device rounds i = 2, 3 exactly and flags the values the library's pow may
// round the other way (exact_power.hpp), whose powers the host then supplies.
// Work proceeds in chunks of elements, so the scratch stays bounded.
void stencil_transforms_device(const TriTopology &mesh, int p,
                               const std::vector<std::int32_t> &neighbors,
                               const std::vector<std::int32_t> &order, const double *d_maps,
                               double *d_transforms, cudaStream_t s);

} // namespace wasl_b200
