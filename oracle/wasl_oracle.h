/*
 * wasl_oracle.h -- CPU restatement of the Wasl modal RKDG hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * product in wasl_b200/: it is imported by tests/, by __graft_entry__.smoke()
 * and by the cpu_baseline leg of bench.py, never by the product itself.
 *
 * Every function restates, in plain C with the same floating-point operation
 * order, one function of the reference solver (indrow/wasl, C++20).  The
 * reference file:line it follows is cited beside each declaration.  Build with
 * -O2 -ffp-contract=off (no FMA contraction) so results are bit-identical to the
 * reference compiled the same way; tests/test_oracle_vs_ref.py checks that
 * against the reference itself built into oracle/_ref, and
 * tests/test_oracle_golden.py against the reference's stored case regression.
 *
 * Layouts follow the reference:
 *   Euler state  U[variable][mode][element]   (cpp/include/wasl/dg/modal_layout.hpp:16-23)
 *   scalar state U[element][mode]             (cpp/include/wasl/dg/scalar_advection/line_residual.hpp:46)
 *   exterior     [variable][face][edge point]  (cpp/include/wasl/dg/euler/triangle_residual.hpp:3-4)
 */
#ifndef WASL_ORACLE_H
#define WASL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- basis (cpp/include/wasl/basis) ---------------------------------- */
double wo_jacobi_p(double x, int n, double alpha, double beta);              /* jacobi.hpp:12-27 */
double wo_jacobi_p_derivative(double x, int n, double alpha, double beta);   /* jacobi.hpp:31-35 */
void wo_legendre_basis(double xi, int p, double *values);                    /* legendre.hpp:23-38 */
void wo_legendre_basis_gradient(double xi, int p, double *gradients);        /* legendre.hpp:41-60 */
void wo_dubiner_basis(double xi, double eta, int p, double *values);         /* dubiner_triangle.hpp:49-63 */
void wo_dubiner_basis_gradient(double xi, double eta, int p, double *gxi,
                               double *geta);                                /* dubiner_triangle.hpp:70-103 */
int wo_line_modes(int p);                                                    /* mode_count.hpp:9 */
int wo_tri_modes(int p);                                                     /* mode_count.hpp:11-13 */

/* ---- quadrature (cpp/include/wasl/quadrature) ------------------------ */
int wo_gauss_legendre(int n, double *points, double *weights);               /* gauss_legendre.hpp:51-65 */
/* (p+1)^2 points; returns the count. triangle_volume_rule.hpp:34-51 */
int wo_tri_volume_rule(int p, double *xi, double *eta, double *weights);
/* 3 edges x (p+1) points, packed [edge][point]; normals [edge]. triangle_edge_rules.hpp:28-58 */
void wo_tri_edge_rules(int p, double *xi, double *eta, double *weights, double *normal_x,
                       double *normal_y);

/* ---- triangle mesh (cpp/src/mesh/triangle/build_triangle_mesh.cpp) ----- */
typedef struct {
  int64_t element_count;
  int64_t face_count;
  double *vertices;       /* [element][6] x0 y0 x1 y1 x2 y2 after orientation */
  int64_t *nodes;         /* [element][3] node tags after orientation */
  int32_t *face_left;     /* [face] */
  int32_t *face_right;    /* [face] -1 on a boundary */
  int32_t *face_left_edge;
  int32_t *face_right_edge;
  int64_t *face_left_v0;  /* vertex each side starts its traversal at */
  int64_t *face_right_v0;
  double *face_normal_x;  /* outward from the left element */
  double *face_normal_y;
} wo_tri_mesh;

/* build_triangle_mesh.cpp:120-148; returns 0 or a negative error code. */
int wo_tri_mesh_build(int64_t node_count, const int64_t *node_tags, const double *node_xy,
                      int64_t element_count, const int64_t *element_nodes, wo_tri_mesh *mesh);
void wo_tri_mesh_free(wo_tri_mesh *mesh);

/* ---- line mesh (cpp/src/mesh/line/build_line_mesh.cpp) ------------------ */
typedef struct {
  int64_t element_count;
  int64_t face_count;
  double *x_left, *x_right;  /* [element] */
  int32_t *face_left, *face_right;
  double *face_x, *face_normal;
} wo_line_mesh;

/* build_line_mesh.cpp:14-84: segments given as node-tag pairs. */
int wo_line_mesh_build(int64_t node_count, const int64_t *node_tags, const double *node_x,
                       int64_t element_count, const int64_t *element_nodes, wo_line_mesh *mesh);
void wo_line_mesh_free(wo_line_mesh *mesh);

/* ---- Euler fluxes (cpp/include/wasl/flux/hllc.hpp:40-74) ---------------- */
void wo_hllc_flux(double gamma, const double *left, const double *right, double nx, double ny,
                  double *flux);

/* ---- residuals (cpp/include/wasl/dg) ------------------------------------ */
/* euler/triangle_residual.hpp:26-107 with hllc_flux */
void wo_euler_tri_residual(const wo_tri_mesh *mesh, double gamma, int p, const double *coefficients,
                           const double *exterior, double *rhs);
/* euler/line_residual.hpp:24-86 with hllc_flux; exterior [variable][face] */
void wo_euler_line_residual(const wo_line_mesh *mesh, double gamma, int p,
                            const double *coefficients, const double *exterior, double *rhs);
/* scalar_advection/line_residual.hpp:48-111, U[element][mode] */
void wo_scalar_line_residual(const wo_line_mesh *mesh, double wavespeed, int p,
                             const double *coefficients, const double *exterior, double *rhs);
/* scalar_advection/triangle_residual.hpp:25-104, U[element][mode], constant velocity */
void wo_scalar_tri_residual(const wo_tri_mesh *mesh, double vx, double vy, int p,
                            const double *coefficients, const double *exterior, double *rhs);

/* ---- exterior traces (cpp/src/boundaries) ------------------------------- */
/* periodic_triangle_trace.cpp:40-67: donors [face][point], basis [face][point][mode].
 * Returns 0 or a negative error (no axis-aligned box / missing donor). */
int wo_periodic_tri_trace(const wo_tri_mesh *mesh, int p, int32_t *donors, double *basis);
/* periodic_triangle_trace.cpp:84-105 */
void wo_periodic_tri_euler_exterior(const wo_tri_mesh *mesh, int p, const int32_t *donors,
                                    const double *basis, const double *coefficients,
                                    double *exterior);
/* periodic_triangle_trace.cpp:69-82, scalar U[element][mode] */
void wo_periodic_tri_scalar_exterior(const wo_tri_mesh *mesh, int p, const int32_t *donors,
                                     const double *basis, const double *coefficients,
                                     double *exterior);
/* Transmissive 2D exterior: the owner's own trace at every boundary edge point.
 * A project extension: the reference has no 2D outflow; this follows the 1D
 * outflow rule line_boundary_conditions.hpp:10-11,47-49. */
void wo_transmissive_tri_euler_exterior(const wo_tri_mesh *mesh, int p, const double *coefficients,
                                        double *exterior);
/* line_euler_exterior.cpp:13-43; kinds 0 periodic, 2 outflow (1 inflow is rejected). */
int wo_line_euler_exterior(const wo_line_mesh *mesh, int p, int left_kind, int right_kind,
                           const double *coefficients, double *exterior);
/* line_boundary_conditions.hpp:36-57 + line_exterior.hpp:17-43, U[element][mode] */
void wo_line_scalar_exterior(const wo_line_mesh *mesh, int p, int left_kind, double left_value,
                             int right_kind, double right_value, const double *coefficients,
                             double *exterior);

/* ---- limiter (cpp/src/limiting) ----------------------------------------- */
typedef struct {
  int64_t element_count;
  int mode_count;
  int polynomial_order;
  int maximum_neighbors;
  int highest_degree_begin;
  int check_point_count;
  int32_t *neighbors;  /* [element][candidate] */
  double *transforms;  /* [element][candidate][target mode][source mode] */
  double *normal_x, *normal_y;
  double *check_basis; /* [point][mode] */
} wo_stencil;

/* euler_limiter_stencil_triangle.cpp:97-112; periodic_donors may be NULL. */
int wo_tri_stencil(const wo_tri_mesh *mesh, int p, const int32_t *periodic_donors,
                   int edge_point_count, wo_stencil *stencil);
/* euler_limiter_stencil_line.cpp:79-94 */
int wo_line_stencil(const wo_line_mesh *mesh, int p, int periodic, wo_stencil *stencil);
void wo_stencil_free(wo_stencil *stencil);
/* euler_modal_limiter.cpp:70-98.  flags (optional, [element]) receives the
 * troubled-cell set.  Returns 0, or -1 where the positivity limiter throws
 * (euler_positivity.hpp:74-75); *bad_element then names the element. */
int wo_limit_euler(const wo_stencil *stencil, double gamma, double threshold, double density_floor,
                   double pressure_floor, double *coefficients, uint8_t *flags,
                   int64_t *bad_element);
/* modal_decay.hpp:23-33 + euler_modal_limiter.cpp:18-24 on every element. */
void wo_troubled_flags(const wo_stencil *stencil, double threshold, const double *coefficients,
                       uint8_t *flags);
/* euler_positivity.hpp:63-102 on one packed [variable][mode] element. */
int wo_positivity(double gamma, double *coefficients, int mode_count, const double *basis,
                  int point_count, double density_floor, double pressure_floor, double *scale);
/* euler_characteristic_weno.hpp:17-67 on one element */
void wo_characteristic_weno(double gamma, const double *average, double nx, double ny,
                            const double *target, const double *candidates, int candidate_count,
                            int mode_count, double *limited);

/* ---- time step (cpp/src/time/cfl_timestep.cpp) -------------------------- */
/* :70-84; returns 0, or -1 on a non-physical cell average (:39-40). */
int wo_euler_tri_cfl(const wo_tri_mesh *mesh, double gamma, const double *coefficients, int p,
                     double cfl, double *dt);
int wo_euler_line_cfl(const wo_line_mesh *mesh, double gamma, const double *coefficients, int p,
                      double cfl, double *dt);
double wo_tri_minimum_altitude(const wo_tri_mesh *mesh);                    /* :22-30 */
double wo_line_advection_cfl(const wo_line_mesh *mesh, double wavespeed, int p, double cfl); /* :55-60 */
double wo_tri_scalar_cfl(const wo_tri_mesh *mesh, double vx, double vy, int p, double cfl);  /* :62-68 */

/* ---- SSP-RK3 (cpp/include/wasl/time/ssp_rk3.hpp:37-61) ------------------- */
/* Boundary kinds for 2D Euler: 0 periodic (donors/basis required), 3 transmissive. */
typedef struct {
  int boundary_kind;
  const int32_t *donors;
  const double *donor_basis;
  const wo_stencil *stencil; /* NULL: no limiting */
  double threshold, density_floor, pressure_floor;
} wo_euler_tri_setup;

/* One step; returns 0 or the limiter error.  flags (optional) receives the
 * troubled set of each of the three stages, packed [stage][element]. */
int wo_euler_tri_step(const wo_tri_mesh *mesh, const wo_euler_tri_setup *setup, double gamma,
                      int p, double dt, double *coefficients, uint8_t *flags);
/* flags (optional, [stage][element]) as for wo_euler_tri_step. */
int wo_euler_line_step(const wo_line_mesh *mesh, int left_kind, int right_kind,
                       const wo_stencil *stencil, double threshold, double density_floor,
                       double pressure_floor, double gamma, int p, double dt,
                       double *coefficients, uint8_t *flags);
void wo_scalar_line_step(const wo_line_mesh *mesh, int left_kind, double left_value,
                         int right_kind, double right_value, double wavespeed, int p, double dt,
                         double *coefficients);
void wo_scalar_tri_step(const wo_tri_mesh *mesh, const int32_t *donors, const double *donor_basis,
                        double vx, double vy, int p, double dt, double *coefficients);

/* ---- projection and diagnostics (cpp/include/wasl/dg/l2_projection.hpp) ------ */
/* Physical points of rule triangle_volume_rule(rule_order) on every element,
 * packed [element][point]. l2_projection.hpp:57-76 (reference_to_physical). */
void wo_tri_rule_points(const wo_tri_mesh *mesh, int rule_order, double *x, double *y);
/* values [element][point][variable] -> U[variable][mode][element] */
void wo_tri_project(const wo_tri_mesh *mesh, int p, int rule_order, int variable_count,
                    const double *values, double *coefficients);
void wo_line_rule_points(const wo_line_mesh *mesh, int point_count, double *x);
void wo_line_project(const wo_line_mesh *mesh, int p, int point_count, int variable_count,
                     const double *values, double *coefficients);
/* euler_diagnostics.cpp:26-39 / scalar_diagnostics.cpp:21-36 */
double wo_tri_mass(const wo_tri_mesh *mesh, const double *mode0, int64_t stride);
double wo_line_mass(const wo_line_mesh *mesh, const double *mode0, int64_t stride);

#ifdef __cplusplus
}
#endif

#endif
