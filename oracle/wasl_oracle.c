/*
 * wasl_oracle.c -- CPU restatement of the Wasl modal RKDG hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA product (see
 * wasl_oracle.h).  Each function follows the reference function cited beside
 * it, written out in C with the same floating-point operation order so that a
 * build with -ffp-contract=off reproduces the reference bit for bit.  Where the
 * reference re-evaluates the same basis value inside a loop this file evaluates
 * it once: the value is a deterministic function of its arguments, so the sums
 * it feeds are unchanged.
 */
#include "wasl_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ====================================================================== */
/* basis                                                                  */
/* ====================================================================== */

/* cpp/include/wasl/basis/jacobi.hpp:12-27 (three-term recurrence, A&S 22.7.1) */
double wo_jacobi_p(double x, int n, double alpha, double beta) {
  if (n <= 0)
    return 1.0;
  double p_prev = 1.0;
  double p_curr = 0.5 * (alpha - beta + (alpha + beta + 2.0) * x);
  for (int k = 1; k < n; ++k) {
    const double ab = 2.0 * k + alpha + beta;
    const double a = 2.0 * (k + 1) * (k + alpha + beta + 1.0) * ab;
    const double b = (ab + 1.0) * (ab * (ab + 2.0) * x + (alpha * alpha - beta * beta));
    const double c = 2.0 * (k + alpha) * (k + beta) * (ab + 2.0);
    const double p_next = (b * p_curr - c * p_prev) / a;
    p_prev = p_curr;
    p_curr = p_next;
  }
  return p_curr;
}

/* jacobi.hpp:31-35 */
double wo_jacobi_p_derivative(double x, int n, double alpha, double beta) {
  if (n <= 0)
    return 0.0;
  return 0.5 * (n + alpha + beta + 1.0) * wo_jacobi_p(x, n - 1, alpha + 1.0, beta + 1.0);
}

static double legendre_norm(int j) { return sqrt((2.0 * j + 1.0) / 2.0); }

/* legendre.hpp:23-38 */
void wo_legendre_basis(double xi, int p, double *values) {
  values[0] = legendre_norm(0);
  if (p <= 0)
    return;
  double p_previous = 1.0;
  double p_current = xi;
  values[1] = legendre_norm(1) * p_current;
  for (int j = 1; j < p; ++j) {
    const double p_next = ((2.0 * j + 1.0) * xi * p_current - j * p_previous) / (j + 1);
    p_previous = p_current;
    p_current = p_next;
    values[j + 1] = legendre_norm(j + 1) * p_current;
  }
}

/* legendre.hpp:41-60 */
void wo_legendre_basis_gradient(double xi, int p, double *gradients) {
  gradients[0] = 0.0;
  if (p <= 0)
    return;
  double p_previous = 1.0, p_current = xi;
  double dp_previous = 0.0, dp_current = 1.0;
  gradients[1] = legendre_norm(1) * dp_current;
  for (int j = 1; j < p; ++j) {
    const double p_next = ((2.0 * j + 1.0) * xi * p_current - j * p_previous) / (j + 1);
    const double dp_next =
        ((2.0 * j + 1.0) * (p_current + xi * dp_current) - j * dp_previous) / (j + 1);
    p_previous = p_current;
    p_current = p_next;
    dp_previous = dp_current;
    dp_current = dp_next;
    gradients[j + 1] = legendre_norm(j + 1) * dp_current;
  }
}

/* dubiner_triangle.hpp:39-41 */
static double collapsed_a(double xi, double eta) {
  return (eta < 1.0) ? (2.0 + 2.0 * xi) / (1.0 - eta) - 1.0 : -1.0;
}

/* dubiner_triangle.hpp:43-45 */
static double dubiner_norm(int i, int n) { return sqrt((2.0 * i + 1.0) * (n + 1.0) / 2.0); }

/* dubiner_triangle.hpp:49-63 */
void wo_dubiner_basis(double xi, double eta, int p, double *values) {
  const double b = eta;
  const double a = collapsed_a(xi, eta);
  const double half_one_minus_b = 0.5 * (1.0 - b);
  int index = 0;
  for (int n = 0; n <= p; ++n) {
    for (int i = 0; i <= n; ++i) {
      const int j = n - i;
      const double pi = wo_jacobi_p(a, i, 0.0, 0.0);
      const double warp = pow(half_one_minus_b, (double)i);
      const double qj = wo_jacobi_p(b, j, 2.0 * i + 1.0, 0.0);
      values[index++] = dubiner_norm(i, n) * pi * warp * qj;
    }
  }
}

/* dubiner_triangle.hpp:70-103 */
void wo_dubiner_basis_gradient(double xi, double eta, int p, double *gxi, double *geta) {
  const double b = eta;
  const double a = collapsed_a(xi, eta);
  const double half_one_minus_b = 0.5 * (1.0 - b);
  const double inverse_one_minus_b = 1.0 / (1.0 - b);
  const double da_dxi = 2.0 * inverse_one_minus_b;
  const double da_deta = (a + 1.0) * inverse_one_minus_b;
  int index = 0;
  for (int n = 0; n <= p; ++n) {
    for (int i = 0; i <= n; ++i) {
      const int j = n - i;
      const double norm = dubiner_norm(i, n);
      const double pi = wo_jacobi_p(a, i, 0.0, 0.0);
      const double warp = pow(half_one_minus_b, (double)i);
      const double qj = wo_jacobi_p(b, j, 2.0 * i + 1.0, 0.0);
      const double dpi_da = wo_jacobi_p_derivative(a, i, 0.0, 0.0);
      const double dqj_db = wo_jacobi_p_derivative(b, j, 2.0 * i + 1.0, 0.0);
      double dwarp_db = 0.0;
      if (i > 0)
        dwarp_db = -0.5 * (double)i * pow(half_one_minus_b, (double)(i - 1));
      const double dphi_da = norm * dpi_da * warp * qj;
      const double dphi_db = norm * (pi * dwarp_db * qj + pi * warp * dqj_db);
      gxi[index] = dphi_da * da_dxi;
      geta[index] = dphi_da * da_deta + dphi_db;
      ++index;
    }
  }
}

int wo_line_modes(int p) { return p + 1; }
int wo_tri_modes(int p) { return (p + 1) * (p + 2) / 2; }

/* ====================================================================== */
/* quadrature                                                             */
/* ====================================================================== */

/* Nonnegative halves of the symmetric Gauss-Legendre rules n = 1..7.  The
 * decimal literals are the reference's tabulation
 * (cpp/include/wasl/quadrature/gauss_legendre.hpp:24-44): the rule values have
 * to be the same doubles for bit-identical sums. */
typedef struct {
  double node, weight;
} gl_half;
static const gl_half gl1[] = {{0.0, 2.0}};
static const gl_half gl2[] = {{0.5773502691896257, 1.0}};
static const gl_half gl3[] = {{0.0, 0.8888888888888888}, {0.7745966692414834, 0.5555555555555556}};
static const gl_half gl4[] = {{0.33998104358485626, 0.6521451548625461},
                              {0.8611363115940526, 0.34785484513745385}};
static const gl_half gl5[] = {{0.0, 0.5688888888888889},
                              {0.5384693101056831, 0.47862867049936647},
                              {0.9061798459386640, 0.2369268850561891}};
static const gl_half gl6[] = {{0.2386191860831969, 0.4679139345726910},
                              {0.6612093864662645, 0.3607615730481386},
                              {0.9324695142031521, 0.17132449237917036}};
static const gl_half gl7[] = {{0.0, 0.4179591836734694},
                              {0.4058451513773972, 0.3818300505051188},
                              {0.7415311855993945, 0.2797053914892766},
                              {0.9491079123427585, 0.1294849661688697}};

/* gauss_legendre.hpp:51-65: mirrored negatives ascending, then the halves. */
int wo_gauss_legendre(int n, double *points, double *weights) {
  static const gl_half *tables[] = {NULL, gl1, gl2, gl3, gl4, gl5, gl6, gl7};
  static const int sizes[] = {0, 1, 1, 2, 2, 3, 3, 4};
  if (n < 1 || n > 7)
    return -1;
  const gl_half *h = tables[n];
  const int count = sizes[n];
  int k = 0;
  for (int i = count - 1; i >= 0; --i) {
    if (h[i].node == 0.0)
      continue;
    points[k] = -h[i].node;
    weights[k] = h[i].weight;
    ++k;
  }
  for (int i = 0; i < count; ++i) {
    points[k] = h[i].node;
    weights[k] = h[i].weight;
    ++k;
  }
  return k;
}

/* triangle_volume_rule.hpp:34-51 */
int wo_tri_volume_rule(int p, double *xi, double *eta, double *weights) {
  const int n = p + 1;
  double pts[8], wts[8];
  wo_gauss_legendre(n, pts, wts);
  int k = 0;
  for (int qb = 0; qb < n; ++qb) {
    const double e = pts[qb];
    const double jacobian = 0.5 * (1.0 - e);
    for (int qa = 0; qa < n; ++qa) {
      const double a = pts[qa];
      xi[k] = 0.5 * (a + 1.0) * (1.0 - e) - 1.0;
      eta[k] = e;
      weights[k] = wts[qb] * wts[qa] * jacobian;
      ++k;
    }
  }
  return k;
}

/* triangle_edge_rules.hpp:28-58 */
void wo_tri_edge_rules(int p, double *xi, double *eta, double *weights, double *normal_x,
                       double *normal_y) {
  const int n = p + 1;
  double pts[8], wts[8];
  wo_gauss_legendre(n, pts, wts);
  const double inverse_sqrt2 = 1.0 / sqrt(2.0);
  normal_x[0] = 0.0;
  normal_y[0] = -1.0;
  normal_x[1] = inverse_sqrt2;
  normal_y[1] = inverse_sqrt2;
  normal_x[2] = -1.0;
  normal_y[2] = 0.0;
  for (int q = 0; q < n; ++q) {
    const double s = pts[q];
    const double weight = wts[q];
    xi[q] = s;
    eta[q] = -1.0;
    weights[q] = weight;
    xi[n + q] = 1.0 + 0.5 * (s + 1.0) * (-2.0);
    eta[n + q] = -1.0 + 0.5 * (s + 1.0) * (2.0);
    weights[n + q] = weight * 2.0 * inverse_sqrt2;
    xi[2 * n + q] = -1.0;
    eta[2 * n + q] = s;
    weights[2 * n + q] = weight;
  }
}

/* ====================================================================== */
/* triangle geometry (cpp/include/wasl/mesh/triangle/triangle_geometry.hpp) */
/* ====================================================================== */

typedef struct {
  double x0, y0, x1, y1, x2, y2;
} tri_map;

static tri_map element_map(const wo_tri_mesh *mesh, int64_t e) {
  const double *v = mesh->vertices + 6 * e;
  tri_map m = {v[0], v[1], v[2], v[3], v[4], v[5]};
  return m;
}
static double map_ax(const tri_map *m) { return m->x1 - m->x0; }
static double map_ay(const tri_map *m) { return m->y1 - m->y0; }
static double map_bx(const tri_map *m) { return m->x2 - m->x0; }
static double map_by(const tri_map *m) { return m->y2 - m->y0; }
/* :39 */
static double map_det_a(const tri_map *m) {
  return map_ax(m) * map_by(m) - map_bx(m) * map_ay(m);
}
/* :42 */
static double map_jacobian_determinant(const tri_map *m) { return map_det_a(m) / 4.0; }
/* :47 */
static int map_orientation(const tri_map *m) { return map_det_a(m) > 0.0 ? 1 : -1; }
/* :49-52 */
static void map_reference_to_physical(const tri_map *m, double xi, double eta, double *x,
                                      double *y) {
  *x = m->x0 + 0.5 * (map_ax(m) * (xi + 1.0) + map_bx(m) * (eta + 1.0));
  *y = m->y0 + 0.5 * (map_ay(m) * (xi + 1.0) + map_by(m) * (eta + 1.0));
}
/* :55-64 */
static void map_physical_to_reference(const tri_map *m, double x, double y, double *xi,
                                      double *eta) {
  const double dx = x - m->x0;
  const double dy = y - m->y0;
  const double inverse_det = 1.0 / map_det_a(m);
  const double s = (map_by(m) * dx - map_bx(m) * dy) * inverse_det;
  const double t = (-map_ay(m) * dx + map_ax(m) * dy) * inverse_det;
  *xi = 2.0 * s - 1.0;
  *eta = 2.0 * t - 1.0;
}
/* :68-72 */
static void map_scaled_gradient(const tri_map *m, double gxi, double geta, double *gx,
                                double *gy) {
  *gx = 0.5 * (map_by(m) * gxi - map_ay(m) * geta);
  *gy = 0.5 * (-map_bx(m) * gxi + map_ax(m) * geta);
}
/* :75-86 */
static void map_edge_vector(const tri_map *m, int edge, double *ex, double *ey) {
  if (edge == 0) {
    *ex = m->x1 - m->x0;
    *ey = m->y1 - m->y0;
  } else if (edge == 1) {
    *ex = m->x2 - m->x1;
    *ey = m->y2 - m->y1;
  } else {
    *ex = m->x0 - m->x2;
    *ey = m->y0 - m->y2;
  }
}
/* :88-92 */
static double map_edge_length(const tri_map *m, int edge) {
  double ex = 0.0, ey = 0.0;
  map_edge_vector(m, edge, &ex, &ey);
  return hypot(ex, ey);
}
/* :96-105 */
static void map_edge_normal(const tri_map *m, int edge, double *nx, double *ny) {
  double ex = 0.0, ey = 0.0;
  map_edge_vector(m, edge, &ex, &ey);
  const double length = hypot(ex, ey);
  const double tx = ex / length;
  const double ty = ey / length;
  const int sign = map_orientation(m);
  *nx = sign * ty;
  *ny = sign * (-tx);
}
/* :24-26 */
static double reference_edge_length(int edge) { return edge == 1 ? 2.0 * sqrt(2.0) : 2.0; }
/* cpp/include/wasl/dg/triangle_face_trace.hpp:36-38 */
static double face_edge_scale(const tri_map *left, int left_edge) {
  return map_edge_length(left, left_edge) / reference_edge_length(left_edge);
}

/* triangle_face_trace.hpp:16-33 */
static void neighbor_edge_point(const wo_tri_mesh *mesh, int64_t f, double lxi, double leta,
                                double *rxi, double *reta) {
  const int le = mesh->face_left_edge[f];
  double parameter = le == 0 ? lxi : le == 1 ? leta : -leta;
  if (mesh->face_left_v0[f] != mesh->face_right_v0[f])
    parameter = -parameter;
  *rxi = -1.0;
  *reta = -1.0;
  const int re = mesh->face_right_edge[f];
  if (re == 0) {
    *rxi = parameter;
  } else if (re == 1) {
    *rxi = -parameter;
    *reta = parameter;
  } else {
    *reta = -parameter;
  }
}

/* ====================================================================== */
/* triangle mesh topology (cpp/src/mesh/triangle/build_triangle_mesh.cpp)  */
/* ====================================================================== */

typedef struct {
  int64_t key_a, key_b;
  int32_t element;
  int32_t local_edge;
  int64_t v0, v1;
} half_edge;

static int compare_half_edge(const void *pa, const void *pb) {
  const half_edge *a = (const half_edge *)pa, *b = (const half_edge *)pb;
  if (a->key_a != b->key_a)
    return a->key_a < b->key_a ? -1 : 1;
  if (a->key_b != b->key_b)
    return a->key_b < b->key_b ? -1 : 1;
  /* first-encountered side first: element, then local edge */
  if (a->element != b->element)
    return a->element < b->element ? -1 : 1;
  return a->local_edge < b->local_edge ? -1 : (a->local_edge > b->local_edge);
}

typedef struct {
  int64_t tag;
  int64_t index;
} tag_index;

static int compare_tag(const void *pa, const void *pb) {
  const tag_index *a = (const tag_index *)pa, *b = (const tag_index *)pb;
  return a->tag < b->tag ? -1 : (a->tag > b->tag);
}

static int64_t lookup_tag(const tag_index *sorted, int64_t count, int64_t tag) {
  int64_t lo = 0, hi = count - 1;
  while (lo <= hi) {
    const int64_t mid = (lo + hi) / 2;
    if (sorted[mid].tag == tag)
      return sorted[mid].index;
    if (sorted[mid].tag < tag)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return -1;
}

typedef struct {
  int32_t left, right, le, re;
  int64_t lv0, rv0;
} face_rec;

static int compare_face(const void *pa, const void *pb) {
  const face_rec *a = (const face_rec *)pa, *b = (const face_rec *)pb;
  if (a->left != b->left)
    return a->left < b->left ? -1 : 1;
  return a->le < b->le ? -1 : (a->le > b->le);
}

static const int triangle_edge_vertices[3][2] = {{0, 1}, {1, 2}, {2, 0}};

/* build_triangle_mesh.cpp:120-148 (oriented_elements :38-65, edge_adjacency
 * :67-90, make_face :94-116, face sort :137-140). */
int wo_tri_mesh_build(int64_t node_count, const int64_t *node_tags, const double *node_xy,
                      int64_t element_count, const int64_t *element_nodes, wo_tri_mesh *mesh) {
  memset(mesh, 0, sizeof(*mesh));
  if (element_count <= 0)
    return -1;
  tag_index *lookup = (tag_index *)malloc(sizeof(tag_index) * (size_t)node_count);
  for (int64_t i = 0; i < node_count; ++i) {
    lookup[i].tag = node_tags[i];
    lookup[i].index = i;
  }
  qsort(lookup, (size_t)node_count, sizeof(tag_index), compare_tag);
  for (int64_t i = 1; i < node_count; ++i)
    if (lookup[i].tag == lookup[i - 1].tag) {
      free(lookup);
      return -2; /* duplicate node tag */
    }

  mesh->element_count = element_count;
  mesh->vertices = (double *)malloc(sizeof(double) * 6 * (size_t)element_count);
  mesh->nodes = (int64_t *)malloc(sizeof(int64_t) * 3 * (size_t)element_count);
  for (int64_t e = 0; e < element_count; ++e) {
    int64_t tags[3];
    double x[3], y[3];
    for (int k = 0; k < 3; ++k) {
      tags[k] = element_nodes[3 * e + k];
      const int64_t idx = lookup_tag(lookup, node_count, tags[k]);
      if (idx < 0) {
        free(lookup);
        wo_tri_mesh_free(mesh);
        return -3; /* missing node */
      }
      x[k] = node_xy[2 * idx];
      y[k] = node_xy[2 * idx + 1];
    }
    const double signed_double_area =
        x[0] * (y[1] - y[2]) + x[1] * (y[2] - y[0]) + x[2] * (y[0] - y[1]);
    if (signed_double_area == 0.0) {
      free(lookup);
      wo_tri_mesh_free(mesh);
      return -4; /* zero-area element */
    }
    if (signed_double_area < 0.0) {
      double t = x[1];
      x[1] = x[2];
      x[2] = t;
      t = y[1];
      y[1] = y[2];
      y[2] = t;
      const int64_t tt = tags[1];
      tags[1] = tags[2];
      tags[2] = tt;
    }
    double *v = mesh->vertices + 6 * e;
    v[0] = x[0];
    v[1] = y[0];
    v[2] = x[1];
    v[3] = y[1];
    v[4] = x[2];
    v[5] = y[2];
    mesh->nodes[3 * e] = tags[0];
    mesh->nodes[3 * e + 1] = tags[1];
    mesh->nodes[3 * e + 2] = tags[2];
  }
  free(lookup);

  const int64_t half_count = 3 * element_count;
  half_edge *halves = (half_edge *)malloc(sizeof(half_edge) * (size_t)half_count);
  for (int64_t e = 0; e < element_count; ++e)
    for (int k = 0; k < 3; ++k) {
      half_edge *h = halves + 3 * e + k;
      h->element = (int32_t)e;
      h->local_edge = k;
      h->v0 = mesh->nodes[3 * e + triangle_edge_vertices[k][0]];
      h->v1 = mesh->nodes[3 * e + triangle_edge_vertices[k][1]];
      h->key_a = h->v0 < h->v1 ? h->v0 : h->v1;
      h->key_b = h->v0 < h->v1 ? h->v1 : h->v0;
    }
  qsort(halves, (size_t)half_count, sizeof(half_edge), compare_half_edge);

  face_rec *faces = (face_rec *)malloc(sizeof(face_rec) * (size_t)half_count);
  int64_t face_count = 0;
  for (int64_t i = 0; i < half_count;) {
    int64_t j = i + 1;
    while (j < half_count && halves[j].key_a == halves[i].key_a &&
           halves[j].key_b == halves[i].key_b)
      ++j;
    if (j - i > 2) {
      free(halves);
      free(faces);
      wo_tri_mesh_free(mesh);
      return -5; /* non-conforming edge */
    }
    face_rec *f = faces + face_count++;
    f->left = halves[i].element;
    f->le = halves[i].local_edge;
    f->lv0 = halves[i].v0;
    if (j - i == 2) {
      f->right = halves[i + 1].element;
      f->re = halves[i + 1].local_edge;
      f->rv0 = halves[i + 1].v0;
    } else {
      f->right = -1;
      f->re = 0;
      f->rv0 = 0;
    }
    i = j;
  }
  free(halves);
  qsort(faces, (size_t)face_count, sizeof(face_rec), compare_face);

  mesh->face_count = face_count;
  mesh->face_left = (int32_t *)malloc(sizeof(int32_t) * (size_t)face_count);
  mesh->face_right = (int32_t *)malloc(sizeof(int32_t) * (size_t)face_count);
  mesh->face_left_edge = (int32_t *)malloc(sizeof(int32_t) * (size_t)face_count);
  mesh->face_right_edge = (int32_t *)malloc(sizeof(int32_t) * (size_t)face_count);
  mesh->face_left_v0 = (int64_t *)malloc(sizeof(int64_t) * (size_t)face_count);
  mesh->face_right_v0 = (int64_t *)malloc(sizeof(int64_t) * (size_t)face_count);
  mesh->face_normal_x = (double *)malloc(sizeof(double) * (size_t)face_count);
  mesh->face_normal_y = (double *)malloc(sizeof(double) * (size_t)face_count);
  for (int64_t f = 0; f < face_count; ++f) {
    mesh->face_left[f] = faces[f].left;
    mesh->face_right[f] = faces[f].right;
    mesh->face_left_edge[f] = faces[f].le;
    mesh->face_right_edge[f] = faces[f].re;
    mesh->face_left_v0[f] = faces[f].lv0;
    mesh->face_right_v0[f] = faces[f].rv0;
    const tri_map m = element_map(mesh, faces[f].left);
    map_edge_normal(&m, faces[f].le, mesh->face_normal_x + f, mesh->face_normal_y + f);
  }
  free(faces);
  return 0;
}

void wo_tri_mesh_free(wo_tri_mesh *mesh) {
  free(mesh->vertices);
  free(mesh->nodes);
  free(mesh->face_left);
  free(mesh->face_right);
  free(mesh->face_left_edge);
  free(mesh->face_right_edge);
  free(mesh->face_left_v0);
  free(mesh->face_right_v0);
  free(mesh->face_normal_x);
  free(mesh->face_normal_y);
  memset(mesh, 0, sizeof(*mesh));
}

/* ====================================================================== */
/* line mesh topology (cpp/src/mesh/line/build_line_mesh.cpp)              */
/* ====================================================================== */

typedef struct {
  int64_t left_node, right_node;
  double x_left, x_right;
  int64_t order;
} line_rec;

static int compare_line(const void *pa, const void *pb) {
  const line_rec *a = (const line_rec *)pa, *b = (const line_rec *)pb;
  if (a->x_left != b->x_left)
    return a->x_left < b->x_left ? -1 : 1;
  /* stable_sort: keep input order among equal keys */
  return a->order < b->order ? -1 : (a->order > b->order);
}

/* build_line_mesh.cpp:14-84 */
int wo_line_mesh_build(int64_t node_count, const int64_t *node_tags, const double *node_x,
                       int64_t element_count, const int64_t *element_nodes, wo_line_mesh *mesh) {
  memset(mesh, 0, sizeof(*mesh));
  if (element_count <= 0)
    return -1;
  tag_index *lookup = (tag_index *)malloc(sizeof(tag_index) * (size_t)node_count);
  for (int64_t i = 0; i < node_count; ++i) {
    lookup[i].tag = node_tags[i];
    lookup[i].index = i;
  }
  qsort(lookup, (size_t)node_count, sizeof(tag_index), compare_tag);
  line_rec *recs = (line_rec *)malloc(sizeof(line_rec) * (size_t)element_count);
  for (int64_t e = 0; e < element_count; ++e) {
    const int64_t a = lookup_tag(lookup, node_count, element_nodes[2 * e]);
    const int64_t b = lookup_tag(lookup, node_count, element_nodes[2 * e + 1]);
    if (a < 0 || b < 0 || node_x[a] == node_x[b]) {
      free(lookup);
      free(recs);
      return -3;
    }
    const int forward = node_x[a] < node_x[b];
    const int64_t l = forward ? a : b, r = forward ? b : a;
    recs[e].left_node = node_tags[l];
    recs[e].right_node = node_tags[r];
    recs[e].x_left = node_x[l];
    recs[e].x_right = node_x[r];
    recs[e].order = e;
  }
  free(lookup);
  qsort(recs, (size_t)element_count, sizeof(line_rec), compare_line);
  for (int64_t i = 0; i + 1 < element_count; ++i)
    if (recs[i].right_node != recs[i + 1].left_node) {
      free(recs);
      return -6; /* gap */
    }
  mesh->element_count = element_count;
  mesh->face_count = element_count + 1;
  mesh->x_left = (double *)malloc(sizeof(double) * (size_t)element_count);
  mesh->x_right = (double *)malloc(sizeof(double) * (size_t)element_count);
  for (int64_t e = 0; e < element_count; ++e) {
    mesh->x_left[e] = recs[e].x_left;
    mesh->x_right[e] = recs[e].x_right;
  }
  free(recs);
  const int64_t F = mesh->face_count;
  mesh->face_left = (int32_t *)malloc(sizeof(int32_t) * (size_t)F);
  mesh->face_right = (int32_t *)malloc(sizeof(int32_t) * (size_t)F);
  mesh->face_x = (double *)malloc(sizeof(double) * (size_t)F);
  mesh->face_normal = (double *)malloc(sizeof(double) * (size_t)F);
  mesh->face_left[0] = 0;
  mesh->face_right[0] = -1;
  mesh->face_x[0] = mesh->x_left[0];
  mesh->face_normal[0] = -1.0;
  for (int64_t i = 0; i + 1 < element_count; ++i) {
    mesh->face_left[i + 1] = (int32_t)i;
    mesh->face_right[i + 1] = (int32_t)(i + 1);
    mesh->face_x[i + 1] = mesh->x_right[i];
    mesh->face_normal[i + 1] = 1.0;
  }
  mesh->face_left[F - 1] = (int32_t)(element_count - 1);
  mesh->face_right[F - 1] = -1;
  mesh->face_x[F - 1] = mesh->x_right[element_count - 1];
  mesh->face_normal[F - 1] = 1.0;
  return 0;
}

void wo_line_mesh_free(wo_line_mesh *mesh) {
  free(mesh->x_left);
  free(mesh->x_right);
  free(mesh->face_left);
  free(mesh->face_right);
  free(mesh->face_x);
  free(mesh->face_normal);
  memset(mesh, 0, sizeof(*mesh));
}

/* cpp/include/wasl/mesh/line/line_geometry.hpp:274-279 */
static double line_jacobian(double xl, double xr) { return (xr - xl) / 2.0; }
static double line_centre(double xl, double xr) { return (xl + xr) / 2.0; }
static double line_to_physical(double xl, double xr, double xi) {
  return line_centre(xl, xr) + line_jacobian(xl, xr) * xi;
}
static double line_to_reference(double xl, double xr, double x) {
  return (x - line_centre(xl, xr)) / line_jacobian(xl, xr);
}

/* ====================================================================== */
/* Euler equation (cpp/include/wasl/equations/euler)                      */
/* ====================================================================== */

typedef struct {
  double rho, vx, vy, p;
} prim_t;

/* primitive.hpp:19-27 */
static prim_t primitive(double gamma, const double *s) {
  const double inverse_density = 1.0 / s[0];
  const double vx = s[1] * inverse_density;
  const double vy = s[2] * inverse_density;
  const double kinetic_energy = 0.5 * (s[1] * vx + s[2] * vy);
  prim_t r = {s[0], vx, vy, (gamma - 1.0) * (s[3] - kinetic_energy)};
  return r;
}
/* primitive.hpp:29-31 */
static double sound_speed(double gamma, const prim_t *v) {
  return sqrt(gamma * v->p / v->rho);
}
/* primitive.hpp:33-36 */
static double normal_velocity(const prim_t *v, double nx, double ny) {
  return v->vx * nx + v->vy * ny;
}
/* flux.hpp:11-16 */
static void flux_x(double gamma, const double *s, double *f) {
  const prim_t v = primitive(gamma, s);
  f[0] = s[1];
  f[1] = s[1] * v.vx + v.p;
  f[2] = s[2] * v.vx;
  f[3] = (s[3] + v.p) * v.vx;
}
/* flux.hpp:18-23 */
static void flux_y(double gamma, const double *s, double *f) {
  const prim_t v = primitive(gamma, s);
  f[0] = s[2];
  f[1] = s[1] * v.vy;
  f[2] = s[2] * v.vy + v.p;
  f[3] = (s[3] + v.p) * v.vy;
}
/* flux.hpp:25-33 */
static void normal_flux(double gamma, const double *s, double nx, double ny, double *f) {
  double fx[4], fy[4];
  flux_x(gamma, s, fx);
  flux_y(gamma, s, fy);
  for (int v = 0; v < 4; ++v)
    f[v] = nx * fx[v] + ny * fy[v];
}
static double std_min(double a, double b) { return (b < a) ? b : a; }
static double std_max(double a, double b) { return (a < b) ? b : a; }

/* hllc.hpp:12-27 */
static void hllc_star_state(const double *s, const prim_t *v, double nx, double ny, double wave,
                            double contact, double *star) {
  const double velocity = normal_velocity(v, nx, ny);
  const double star_density = s[0] * (wave - velocity) / (wave - contact);
  const double velocity_shift = contact - velocity;
  const double specific_star_energy =
      s[3] / s[0] + velocity_shift * (contact + v->p / (s[0] * (wave - velocity)));
  star[0] = star_density;
  star[1] = star_density * (v->vx + velocity_shift * nx);
  star[2] = star_density * (v->vy + velocity_shift * ny);
  star[3] = star_density * specific_star_energy;
}

/* hllc.hpp:40-74 (+ add_scaled_jump :29-35) */
void wo_hllc_flux(double gamma, const double *left, const double *right, double nx, double ny,
                  double *flux) {
  const prim_t lv = primitive(gamma, left);
  const prim_t rv = primitive(gamma, right);
  const double lu = normal_velocity(&lv, nx, ny);
  const double ru = normal_velocity(&rv, nx, ny);
  const double lc = sound_speed(gamma, &lv);
  const double rc = sound_speed(gamma, &rv);
  const double left_wave = std_min(lu - lc, ru - rc);
  const double right_wave = std_max(lu + lc, ru + rc);
  double lf[4];
  normal_flux(gamma, left, nx, ny, lf);
  if (left_wave >= 0.0) {
    memcpy(flux, lf, sizeof(lf));
    return;
  }
  double rf[4];
  normal_flux(gamma, right, nx, ny, rf);
  if (right_wave <= 0.0) {
    memcpy(flux, rf, sizeof(rf));
    return;
  }
  const double contact = (rv.p - lv.p + left[0] * lu * (left_wave - lu) -
                          right[0] * ru * (right_wave - ru)) /
                         (left[0] * (left_wave - lu) - right[0] * (right_wave - ru));
  double star[4];
  if (contact >= 0.0) {
    hllc_star_state(left, &lv, nx, ny, left_wave, contact, star);
    for (int v = 0; v < 4; ++v)
      flux[v] = lf[v] + left_wave * (star[v] - left[v]);
    return;
  }
  hllc_star_state(right, &rv, nx, ny, right_wave, contact, star);
  for (int v = 0; v < 4; ++v)
    flux[v] = rf[v] + right_wave * (star[v] - right[v]);
}

/* modal_layout.hpp:26-36: sum in mode order from 0.0 */
static void evaluate_state(const double *c, int M, int64_t ne, int64_t e, const double *basis,
                           double *state) {
  for (int v = 0; v < 4; ++v) {
    double s = 0.0;
    for (int m = 0; m < M; ++m)
      s += c[((int64_t)v * M + m) * ne + e] * basis[m];
    state[v] = s;
  }
}

/* modal_expansion.hpp:14-20 */
static double modal_sum(const double *c, const double *b, int M) {
  double value = 0.0;
  for (int m = 0; m < M; ++m)
    value += c[m] * b[m];
  return value;
}

/* ====================================================================== */
/* residuals                                                              */
/* ====================================================================== */

#define MAXM 36 /* modes up to P7 lines / P6 triangles */
#define MAXQ 100

/* cpp/include/wasl/dg/euler/triangle_residual.hpp:26-107 */
void wo_euler_tri_residual(const wo_tri_mesh *mesh, double gamma, int p, const double *c,
                           const double *exterior, double *rhs) {
  const int M = wo_tri_modes(p);
  const int64_t ne = mesh->element_count, F = mesh->face_count;
  const int Qf = p + 1;
  double vxi[MAXQ], veta[MAXQ], vw[MAXQ];
  const int Qv = wo_tri_volume_rule(p + 2, vxi, veta, vw);
  double exi[3 * 8], eeta[3 * 8], ew[3 * 8], enx[3], eny[3];
  wo_tri_edge_rules(p, exi, eeta, ew, enx, eny);
  memset(rhs, 0, sizeof(double) * 4 * (size_t)M * (size_t)ne);

  static double basis[MAXQ][MAXM], gxi[MAXQ][MAXM], geta[MAXQ][MAXM];
  for (int q = 0; q < Qv; ++q) {
    wo_dubiner_basis(vxi[q], veta[q], p, basis[q]);
    wo_dubiner_basis_gradient(vxi[q], veta[q], p, gxi[q], geta[q]);
  }
  for (int64_t e = 0; e < ne; ++e) {
    const tri_map map = element_map(mesh, e);
    for (int q = 0; q < Qv; ++q) {
      double state[4], fx[4], fy[4];
      evaluate_state(c, M, ne, e, basis[q], state);
      flux_x(gamma, state, fx);
      flux_y(gamma, state, fy);
      for (int m = 0; m < M; ++m) {
        double gx = 0.0, gy = 0.0;
        map_scaled_gradient(&map, gxi[q][m], geta[q][m], &gx, &gy);
        for (int v = 0; v < 4; ++v)
          rhs[((int64_t)v * M + m) * ne + e] += vw[q] * (fx[v] * gx + fy[v] * gy);
      }
    }
  }

  double lb[MAXM], rb[MAXM];
  for (int64_t f = 0; f < F; ++f) {
    const int64_t left = mesh->face_left[f];
    const int le = mesh->face_left_edge[f];
    const tri_map lmap = element_map(mesh, left);
    const double edge_scale = face_edge_scale(&lmap, le);
    const int boundary = mesh->face_right[f] < 0;
    for (int q = 0; q < Qf; ++q) {
      const double lxi = exi[le * Qf + q], leta = eeta[le * Qf + q];
      wo_dubiner_basis(lxi, leta, p, lb);
      double ls[4], rs[4] = {0.0, 0.0, 0.0, 0.0}, flux[4];
      evaluate_state(c, M, ne, left, lb, ls);
      if (!boundary) {
        double rxi = 0.0, reta = 0.0;
        neighbor_edge_point(mesh, f, lxi, leta, &rxi, &reta);
        wo_dubiner_basis(rxi, reta, p, rb);
        evaluate_state(c, M, ne, mesh->face_right[f], rb, rs);
      } else {
        for (int v = 0; v < 4; ++v)
          rs[v] = exterior[((int64_t)v * F + f) * Qf + q];
      }
      wo_hllc_flux(gamma, ls, rs, mesh->face_normal_x[f], mesh->face_normal_y[f], flux);
      const double weight = ew[le * Qf + q] * edge_scale;
      for (int v = 0; v < 4; ++v) {
        const double value = flux[v] * weight;
        for (int m = 0; m < M; ++m)
          rhs[((int64_t)v * M + m) * ne + left] -= value * lb[m];
        if (!boundary) {
          const int64_t right = mesh->face_right[f];
          for (int m = 0; m < M; ++m)
            rhs[((int64_t)v * M + m) * ne + right] += value * rb[m];
        }
      }
    }
  }
  /* modal_layout.hpp:50-56 */
  for (int64_t e = 0; e < ne; ++e) {
    const tri_map map = element_map(mesh, e);
    const double factor = 1.0 / map_jacobian_determinant(&map);
    for (int v = 0; v < 4; ++v)
      for (int m = 0; m < M; ++m)
        rhs[((int64_t)v * M + m) * ne + e] *= factor;
  }
}

/* cpp/include/wasl/dg/euler/line_residual.hpp:24-86 */
void wo_euler_line_residual(const wo_line_mesh *mesh, double gamma, int p, const double *c,
                            const double *exterior, double *rhs) {
  const int M = wo_line_modes(p);
  const int64_t ne = mesh->element_count, F = mesh->face_count;
  double pts[8], wts[8];
  const int nq = wo_gauss_legendre(p + 1 > 1 ? p + 1 : 1, pts, wts);
  memset(rhs, 0, sizeof(double) * 4 * (size_t)M * (size_t)ne);
  double basis[8][MAXM], grad[8][MAXM];
  for (int q = 0; q < nq; ++q) {
    wo_legendre_basis(pts[q], p, basis[q]);
    wo_legendre_basis_gradient(pts[q], p, grad[q]);
  }
  for (int64_t e = 0; e < ne; ++e)
    for (int q = 0; q < nq; ++q) {
      double state[4], f[4];
      evaluate_state(c, M, ne, e, basis[q], state);
      flux_x(gamma, state, f);
      for (int v = 0; v < 4; ++v)
        for (int m = 0; m < M; ++m)
          rhs[((int64_t)v * M + m) * ne + e] += wts[q] * f[v] * grad[q][m];
    }
  double lb[MAXM], rb[MAXM];
  wo_legendre_basis(-1.0, p, lb);
  wo_legendre_basis(1.0, p, rb);
  for (int64_t fi = 0; fi < F; ++fi) {
    const int64_t left = mesh->face_left[fi];
    const int owned_at_left_end = mesh->face_normal[fi] < 0.0;
    const double *ob = owned_at_left_end ? lb : rb;
    double owner[4], ext[4] = {0.0, 0.0, 0.0, 0.0}, flux[4];
    evaluate_state(c, M, ne, left, ob, owner);
    const int boundary = mesh->face_right[fi] < 0;
    if (!boundary) {
      evaluate_state(c, M, ne, mesh->face_right[fi], lb, ext);
    } else {
      for (int v = 0; v < 4; ++v)
        ext[v] = exterior[(int64_t)v * F + fi];
    }
    if (owned_at_left_end)
      wo_hllc_flux(gamma, ext, owner, 1.0, 0.0, flux);
    else
      wo_hllc_flux(gamma, owner, ext, 1.0, 0.0, flux);
    for (int v = 0; v < 4; ++v) {
      const double value = flux[v];
      for (int m = 0; m < M; ++m)
        rhs[((int64_t)v * M + m) * ne + left] += (owned_at_left_end ? 1.0 : -1.0) * ob[m] * value;
      if (!boundary) {
        const int64_t right = mesh->face_right[fi];
        for (int m = 0; m < M; ++m)
          rhs[((int64_t)v * M + m) * ne + right] += lb[m] * value;
      }
    }
  }
  for (int64_t e = 0; e < ne; ++e) {
    const double factor = 1.0 / line_jacobian(mesh->x_left[e], mesh->x_right[e]);
    for (int v = 0; v < 4; ++v)
      for (int m = 0; m < M; ++m)
        rhs[((int64_t)v * M + m) * ne + e] *= factor;
  }
}

/* cpp/include/wasl/equations/scalar_advection/scalar_advection.hpp:36-42 */
static double upwind_flux(double a, double l, double r) { return a >= 0.0 ? a * l : a * r; }

/* cpp/include/wasl/dg/scalar_advection/line_residual.hpp:48-111 */
void wo_scalar_line_residual(const wo_line_mesh *mesh, double a, int p, const double *c,
                             const double *exterior, double *rhs) {
  const int M = wo_line_modes(p);
  const int64_t ne = mesh->element_count, F = mesh->face_count;
  double pts[8], wts[8];
  const int nq = wo_gauss_legendre(p > 0 ? p : 1, pts, wts);
  memset(rhs, 0, sizeof(double) * (size_t)M * (size_t)ne);
  double basis[8][MAXM], grad[8][MAXM];
  for (int q = 0; q < nq; ++q) {
    wo_legendre_basis(pts[q], p, basis[q]);
    wo_legendre_basis_gradient(pts[q], p, grad[q]);
  }
  for (int64_t e = 0; e < ne; ++e) {
    const double *modes = c + e * M;
    double *er = rhs + e * M;
    for (int q = 0; q < nq; ++q) {
      const double flux = a * modal_sum(modes, basis[q], M);
      for (int m = 0; m < M; ++m)
        er[m] += wts[q] * flux * grad[q][m];
    }
  }
  double bl[MAXM], br[MAXM];
  wo_legendre_basis(-1.0, p, bl);
  wo_legendre_basis(1.0, p, br);
  for (int64_t f = 0; f < F; ++f) {
    const double *lm = c + (int64_t)mesh->face_left[f] * M;
    double *lr = rhs + (int64_t)mesh->face_left[f] * M;
    if (mesh->face_normal[f] > 0.0) {
      const double interior = modal_sum(lm, br, M);
      const double flux = upwind_flux(a, interior, exterior[f]);
      for (int m = 0; m < M; ++m)
        lr[m] -= br[m] * flux;
      if (mesh->face_right[f] >= 0) {
        double *rr = rhs + (int64_t)mesh->face_right[f] * M;
        for (int m = 0; m < M; ++m)
          rr[m] += bl[m] * flux;
      }
    } else {
      const double interior = modal_sum(lm, bl, M);
      const double flux = upwind_flux(a, exterior[f], interior);
      for (int m = 0; m < M; ++m)
        lr[m] += bl[m] * flux;
    }
  }
  for (int64_t e = 0; e < ne; ++e) {
    const double inverse_jacobian = 1.0 / line_jacobian(mesh->x_left[e], mesh->x_right[e]);
    for (int m = 0; m < M; ++m)
      rhs[e * M + m] *= inverse_jacobian;
  }
}

/* cpp/include/wasl/dg/scalar_advection/triangle_residual.hpp:25-104 (constant velocity) */
void wo_scalar_tri_residual(const wo_tri_mesh *mesh, double vx, double vy, int p,
                            const double *c, const double *exterior, double *rhs) {
  const int M = wo_tri_modes(p);
  const int64_t ne = mesh->element_count, F = mesh->face_count;
  const int Qf = p + 1;
  double vxi[MAXQ], veta[MAXQ], vw[MAXQ];
  const int Qv = wo_tri_volume_rule(p, vxi, veta, vw);
  double exi[24], eeta[24], ew[24], enx[3], eny[3];
  wo_tri_edge_rules(p, exi, eeta, ew, enx, eny);
  memset(rhs, 0, sizeof(double) * (size_t)M * (size_t)ne);
  static double basis[MAXQ][MAXM], gxi[MAXQ][MAXM], geta[MAXQ][MAXM];
  for (int q = 0; q < Qv; ++q) {
    wo_dubiner_basis(vxi[q], veta[q], p, basis[q]);
    wo_dubiner_basis_gradient(vxi[q], veta[q], p, gxi[q], geta[q]);
  }
  for (int64_t e = 0; e < ne; ++e) {
    const tri_map map = element_map(mesh, e);
    const double *modes = c + e * M;
    double *er = rhs + e * M;
    for (int q = 0; q < Qv; ++q) {
      const double state = modal_sum(modes, basis[q], M);
      for (int m = 0; m < M; ++m) {
        double gx = 0.0, gy = 0.0;
        map_scaled_gradient(&map, gxi[q][m], geta[q][m], &gx, &gy);
        er[m] += vw[q] * state * (vx * gx + vy * gy);
      }
    }
  }
  double lb[MAXM], rb[MAXM];
  for (int64_t f = 0; f < F; ++f) {
    const int64_t left = mesh->face_left[f];
    const int le = mesh->face_left_edge[f];
    const tri_map lmap = element_map(mesh, left);
    const double edge_scale = face_edge_scale(&lmap, le);
    const int boundary = mesh->face_right[f] < 0;
    const double nx = mesh->face_normal_x[f], ny = mesh->face_normal_y[f];
    for (int q = 0; q < Qf; ++q) {
      const double lxi = exi[le * Qf + q], leta = eeta[le * Qf + q];
      wo_dubiner_basis(lxi, leta, p, lb);
      const double ls = modal_sum(c + left * M, lb, M);
      double rs = 0.0;
      if (!boundary) {
        double rxi = 0.0, reta = 0.0;
        neighbor_edge_point(mesh, f, lxi, leta, &rxi, &reta);
        wo_dubiner_basis(rxi, reta, p, rb);
        rs = modal_sum(c + (int64_t)mesh->face_right[f] * M, rb, M);
      } else {
        rs = exterior[f * Qf + q];
      }
      /* scalar_advection.hpp:46-50 */
      const double normal_speed = vx * nx + vy * ny;
      const double flux = normal_speed * (normal_speed >= 0.0 ? ls : rs);
      const double weight = ew[le * Qf + q] * edge_scale;
      double *lr = rhs + left * M;
      for (int m = 0; m < M; ++m)
        lr[m] -= weight * lb[m] * flux;
      if (!boundary) {
        double *rr = rhs + (int64_t)mesh->face_right[f] * M;
        for (int m = 0; m < M; ++m)
          rr[m] += weight * rb[m] * flux;
      }
    }
  }
  for (int64_t e = 0; e < ne; ++e) {
    const tri_map map = element_map(mesh, e);
    const double inverse_mass = 1.0 / map_jacobian_determinant(&map);
    for (int m = 0; m < M; ++m)
      rhs[e * M + m] *= inverse_mass;
  }
}

/* ====================================================================== */
/* exterior traces                                                        */
/* ====================================================================== */

typedef struct {
  double min_x, max_x, min_y, max_y;
} bbox_t;

/* cpp/include/wasl/mesh/triangle/bounding_box.hpp:21-31 */
static bbox_t bounding_box(const wo_tri_mesh *mesh) {
  bbox_t b = {DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
  for (int64_t e = 0; e < mesh->element_count; ++e) {
    const double *v = mesh->vertices + 6 * e;
    for (int k = 0; k < 3; ++k) {
      b.min_x = std_min(b.min_x, v[2 * k]);
      b.max_x = std_max(b.max_x, v[2 * k]);
      b.min_y = std_min(b.min_y, v[2 * k + 1]);
      b.max_y = std_max(b.max_y, v[2 * k + 1]);
    }
  }
  return b;
}

/* periodic_triangle_trace.cpp:28-36: the first element, by index, whose
 * reference coordinates contain the point within 1e-10.  The element bounding
 * box test only skips elements the containment test would reject. */
static int32_t find_donor(const wo_tri_mesh *mesh, double x, double y, double *xi, double *eta) {
  const double tolerance = 1e-10;
  for (int64_t e = 0; e < mesh->element_count; ++e) {
    const double *v = mesh->vertices + 6 * e;
    const double lo_x = std_min(std_min(v[0], v[2]), v[4]), hi_x = std_max(std_max(v[0], v[2]), v[4]);
    const double lo_y = std_min(std_min(v[1], v[3]), v[5]), hi_y = std_max(std_max(v[1], v[3]), v[5]);
    const double margin = 1e-6 * ((hi_x - lo_x) + (hi_y - lo_y));
    if (x < lo_x - margin || x > hi_x + margin || y < lo_y - margin || y > hi_y + margin)
      continue;
    const tri_map m = element_map(mesh, e);
    map_physical_to_reference(&m, x, y, xi, eta);
    if (*xi >= -1.0 - tolerance && *eta >= -1.0 - tolerance && *xi + *eta <= tolerance)
      return (int32_t)e;
  }
  return -1;
}

/* periodic_triangle_trace.cpp:40-67 */
int wo_periodic_tri_trace(const wo_tri_mesh *mesh, int p, int32_t *donors, double *basis) {
  const int M = wo_tri_modes(p);
  const int Q = p + 1;
  double exi[24], eeta[24], ew[24], enx[3], eny[3];
  wo_tri_edge_rules(p, exi, eeta, ew, enx, eny);
  const bbox_t box = bounding_box(mesh);
  for (int64_t i = 0; i < mesh->face_count * Q; ++i)
    donors[i] = -1;
  memset(basis, 0, sizeof(double) * (size_t)(mesh->face_count * Q * M));
  for (int64_t f = 0; f < mesh->face_count; ++f) {
    if (mesh->face_right[f] >= 0)
      continue;
    const tri_map map = element_map(mesh, mesh->face_left[f]);
    const int le = mesh->face_left_edge[f];
    const double nx = mesh->face_normal_x[f], ny = mesh->face_normal_y[f];
    for (int q = 0; q < Q; ++q) {
      double x = 0.0, y = 0.0;
      map_reference_to_physical(&map, exi[le * Q + q], eeta[le * Q + q], &x, &y);
      /* :16-24 periodic_image */
      if (fabs(nx) > 0.5 && fabs(ny) < 1e-10)
        x += nx < 0.0 ? box.max_x - box.min_x : box.min_x - box.max_x;
      else if (fabs(ny) > 0.5 && fabs(nx) < 1e-10)
        y += ny < 0.0 ? box.max_y - box.min_y : box.min_y - box.max_y;
      else
        return -1;
      double xi = 0.0, eta = 0.0;
      const int32_t donor = find_donor(mesh, x, y, &xi, &eta);
      if (donor < 0)
        return -2;
      donors[f * Q + q] = donor;
      wo_dubiner_basis(xi, eta, p, basis + (f * Q + q) * M);
    }
  }
  return 0;
}

/* periodic_triangle_trace.cpp:84-105 */
void wo_periodic_tri_euler_exterior(const wo_tri_mesh *mesh, int p, const int32_t *donors,
                                    const double *basis, const double *c, double *exterior) {
  const int M = wo_tri_modes(p);
  const int Q = p + 1;
  const int64_t F = mesh->face_count, ne = mesh->element_count;
  memset(exterior, 0, sizeof(double) * 4 * (size_t)(F * Q));
  for (int64_t point = 0; point < F * Q; ++point) {
    if (donors[point] < 0)
      continue;
    const int64_t donor = donors[point];
    const int64_t face = point / Q, qp = point % Q;
    for (int v = 0; v < 4; ++v)
      for (int m = 0; m < M; ++m)
        exterior[((int64_t)v * F + face) * Q + qp] +=
            c[((int64_t)v * M + m) * ne + donor] * basis[point * M + m];
  }
}

/* periodic_triangle_trace.cpp:69-82 */
void wo_periodic_tri_scalar_exterior(const wo_tri_mesh *mesh, int p, const int32_t *donors,
                                     const double *basis, const double *c, double *exterior) {
  const int M = wo_tri_modes(p);
  const int Q = p + 1;
  const int64_t F = mesh->face_count;
  memset(exterior, 0, sizeof(double) * (size_t)(F * Q));
  for (int64_t point = 0; point < F * Q; ++point) {
    if (donors[point] < 0)
      continue;
    const int64_t donor = donors[point];
    for (int m = 0; m < M; ++m)
      exterior[point] += c[donor * M + m] * basis[point * M + m];
  }
}

void wo_transmissive_tri_euler_exterior(const wo_tri_mesh *mesh, int p, const double *c,
                                        double *exterior) {
  const int M = wo_tri_modes(p);
  const int Q = p + 1;
  const int64_t F = mesh->face_count, ne = mesh->element_count;
  double exi[24], eeta[24], ew[24], enx[3], eny[3], lb[MAXM];
  wo_tri_edge_rules(p, exi, eeta, ew, enx, eny);
  memset(exterior, 0, sizeof(double) * 4 * (size_t)(F * Q));
  for (int64_t f = 0; f < F; ++f) {
    if (mesh->face_right[f] >= 0)
      continue;
    const int le = mesh->face_left_edge[f];
    for (int q = 0; q < Q; ++q) {
      wo_dubiner_basis(exi[le * Q + q], eeta[le * Q + q], p, lb);
      double s[4];
      evaluate_state(c, M, ne, mesh->face_left[f], lb, s);
      for (int v = 0; v < 4; ++v)
        exterior[((int64_t)v * F + f) * Q + q] = s[v];
    }
  }
}

/* line_euler_exterior.cpp:13-43 */
int wo_line_euler_exterior(const wo_line_mesh *mesh, int p, int left_kind, int right_kind,
                           const double *c, double *exterior) {
  const int M = wo_line_modes(p);
  const int64_t ne = mesh->element_count, F = mesh->face_count;
  double lb[MAXM], rb[MAXM];
  wo_legendre_basis(-1.0, p, lb);
  wo_legendre_basis(1.0, p, rb);
  memset(exterior, 0, sizeof(double) * 4 * (size_t)F);
  for (int64_t f = 0; f < F; ++f) {
    if (mesh->face_right[f] >= 0)
      continue;
    const int left_end = mesh->face_normal[f] < 0.0;
    const int kind = left_end ? left_kind : right_kind;
    if (kind == 1)
      return -1; /* inflow is not implemented for Euler */
    const int periodic = kind == 0;
    const int64_t donor = periodic ? (left_end ? ne - 1 : 0) : mesh->face_left[f];
    const int right_endpoint = periodic ? left_end : !left_end;
    const double *b = right_endpoint ? rb : lb;
    for (int v = 0; v < 4; ++v)
      for (int m = 0; m < M; ++m)
        exterior[(int64_t)v * F + f] += c[((int64_t)v * M + m) * ne + donor] * b[m];
  }
  return 0;
}

/* line_exterior.hpp:17-24 */
static double line_trace(const double *c, int64_t e, int p, double xi) {
  double b[MAXM];
  wo_legendre_basis(xi, p, b);
  return modal_sum(c + e * (p + 1), b, p + 1);
}

/* line_boundary_conditions.hpp:36-57 + line_exterior.hpp:28-43 */
void wo_line_scalar_exterior(const wo_line_mesh *mesh, int p, int left_kind, double left_value,
                             int right_kind, double right_value, const double *c,
                             double *exterior) {
  const int64_t ne = mesh->element_count;
  for (int64_t f = 0; f < mesh->face_count; ++f) {
    if (mesh->face_right[f] >= 0) {
      exterior[f] = line_trace(c, mesh->face_right[f], p, -1.0);
      continue;
    }
    const int left_end = mesh->face_normal[f] < 0.0;
    const int kind = left_end ? left_kind : right_kind;
    if (kind == 1)
      exterior[f] = left_end ? left_value : right_value;
    else if (kind == 2)
      exterior[f] = line_trace(c, mesh->face_left[f], p, left_end ? -1.0 : 1.0);
    else
      exterior[f] = left_end ? line_trace(c, ne - 1, p, 1.0) : line_trace(c, 0, p, -1.0);
  }
}

/* ====================================================================== */
/* limiter stencil                                                        */
/* ====================================================================== */

/* limiter_stencil_assembly.hpp:27-40 */
static void append_unique_neighbor(wo_stencil *s, int64_t element, int32_t neighbor) {
  int32_t *values = s->neighbors + element * s->maximum_neighbors;
  for (int i = 0; i < s->maximum_neighbors; ++i) {
    if (values[i] == neighbor)
      return;
    if (values[i] == -1) {
      values[i] = neighbor;
      return;
    }
  }
}

/* limiter_stencil_assembly.hpp:45-47 */
static double periodic_offset(double gap, double period) {
  return gap > 0.5 * period ? period : gap < -0.5 * period ? -period : 0.0;
}

static void stencil_allocate(wo_stencil *s, int64_t ne, int M, int p, int maxnb) {
  s->element_count = ne;
  s->mode_count = M;
  s->polynomial_order = p;
  s->maximum_neighbors = maxnb;
  s->neighbors = (int32_t *)malloc(sizeof(int32_t) * (size_t)(ne * maxnb));
  for (int64_t i = 0; i < ne * maxnb; ++i)
    s->neighbors[i] = -1;
  s->normal_x = (double *)malloc(sizeof(double) * (size_t)ne);
  s->normal_y = (double *)malloc(sizeof(double) * (size_t)ne);
  for (int64_t e = 0; e < ne; ++e) {
    s->normal_x[e] = 1.0;
    s->normal_y[e] = 0.0;
  }
  s->transforms = (double *)calloc((size_t)(ne * maxnb * M * M), sizeof(double));
}

/* candidate_transform.hpp:18-39 with unit source coefficients */
static void project_neighbor_polynomial(const tri_map *source, const tri_map *target, int p,
                                        const double *sc, double *tc) {
  const int M = wo_tri_modes(p);
  double qxi[MAXQ], qeta[MAXQ], qw[MAXQ], sb[MAXM], tb[MAXM];
  const int Q = wo_tri_volume_rule(p, qxi, qeta, qw);
  for (int m = 0; m < M; ++m)
    tc[m] = 0.0;
  for (int q = 0; q < Q; ++q) {
    double x = 0.0, y = 0.0;
    map_reference_to_physical(target, qxi[q], qeta[q], &x, &y);
    double sxi = 0.0, seta = 0.0;
    map_physical_to_reference(source, x, y, &sxi, &seta);
    wo_dubiner_basis(sxi, seta, p, sb);
    wo_dubiner_basis(qxi[q], qeta[q], p, tb);
    const double value = modal_sum(sc, sb, M);
    for (int m = 0; m < M; ++m)
      tc[m] += qw[q] * value * tb[m];
  }
}

/* euler_limiter_stencil_triangle.cpp:97-112 (connect :16-44, transforms :51-79,
 * check basis :81-93) */
int wo_tri_stencil(const wo_tri_mesh *mesh, int p, const int32_t *periodic_donors,
                   int edge_point_count, wo_stencil *s) {
  memset(s, 0, sizeof(*s));
  const int M = wo_tri_modes(p);
  const int64_t ne = mesh->element_count;
  stencil_allocate(s, ne, M, p, 3);
  s->highest_degree_begin = p > 0 ? wo_tri_modes(p - 1) : M;
  unsigned char *has_normal = (unsigned char *)calloc((size_t)ne, 1);
  for (int64_t f = 0; f < mesh->face_count; ++f) {
    const int64_t left = mesh->face_left[f];
    int32_t right = mesh->face_right[f];
    const int boundary = right < 0;
    if (boundary && periodic_donors)
      right = periodic_donors[f * edge_point_count];
    if (right < 0)
      continue;
    append_unique_neighbor(s, left, right);
    if (!has_normal[left]) {
      s->normal_x[left] = mesh->face_normal_x[f];
      s->normal_y[left] = mesh->face_normal_y[f];
      has_normal[left] = 1;
    }
    if (!boundary) {
      append_unique_neighbor(s, right, (int32_t)left);
      if (!has_normal[right]) {
        s->normal_x[right] = -mesh->face_normal_x[f];
        s->normal_y[right] = -mesh->face_normal_y[f];
        has_normal[right] = 1;
      }
    }
  }
  free(has_normal);

  const bbox_t box = bounding_box(mesh);
  const double width = box.max_x - box.min_x, height = box.max_y - box.min_y;
  double source[MAXM], projected[MAXM];
  for (int m = 0; m < M; ++m)
    source[m] = 0.0;
  for (int64_t e = 0; e < ne; ++e) {
    const tri_map target = element_map(mesh, e);
    for (int k = 0; k < 3; ++k) {
      const int32_t nb = s->neighbors[e * 3 + k];
      if (nb < 0)
        continue;
      tri_map sm = element_map(mesh, nb);
      /* euler_limiter_stencil_triangle.cpp:47-49 centroid_gap */
      const double gx =
          (target.x0 + target.x1 + target.x2 - sm.x0 - sm.x1 - sm.x2) / 3.0;
      const double gy =
          (target.y0 + target.y1 + target.y2 - sm.y0 - sm.y1 - sm.y2) / 3.0;
      const double ox = periodic_offset(gx, width), oy = periodic_offset(gy, height);
      sm.x0 += ox;
      sm.x1 += ox;
      sm.x2 += ox;
      sm.y0 += oy;
      sm.y1 += oy;
      sm.y2 += oy;
      double *matrix = s->transforms + (e * 3 + k) * M * M;
      for (int sm_i = 0; sm_i < M; ++sm_i) {
        source[sm_i] = 1.0;
        project_neighbor_polynomial(&sm, &target, p, source, projected);
        source[sm_i] = 0.0;
        for (int t = 0; t < M; ++t)
          matrix[t * M + sm_i] = projected[t];
      }
    }
  }
  double qxi[MAXQ], qeta[MAXQ], qw[MAXQ];
  const int Qv = wo_tri_volume_rule(p, qxi, qeta, qw);
  double exi[24], eeta[24], ew[24], enx[3], eny[3];
  wo_tri_edge_rules(p, exi, eeta, ew, enx, eny);
  s->check_point_count = Qv + 3 * (p + 1);
  s->check_basis = (double *)malloc(sizeof(double) * (size_t)(s->check_point_count * M));
  for (int q = 0; q < Qv; ++q)
    wo_dubiner_basis(qxi[q], qeta[q], p, s->check_basis + q * M);
  for (int q = 0; q < 3 * (p + 1); ++q)
    wo_dubiner_basis(exi[q], eeta[q], p, s->check_basis + (Qv + q) * M);
  return 0;
}

/* euler_limiter_stencil_line.cpp:79-94 (connect :14-34, transforms :37-63,
 * check basis :65-75) */
int wo_line_stencil(const wo_line_mesh *mesh, int p, int periodic, wo_stencil *s) {
  memset(s, 0, sizeof(*s));
  const int M = wo_line_modes(p);
  const int64_t ne = mesh->element_count;
  stencil_allocate(s, ne, M, p, 2);
  s->highest_degree_begin = p > 0 ? M - 1 : M;
  int32_t left_boundary = -1, right_boundary = -1;
  for (int64_t f = 0; f < mesh->face_count; ++f) {
    if (mesh->face_right[f] >= 0) {
      append_unique_neighbor(s, mesh->face_left[f], mesh->face_right[f]);
      append_unique_neighbor(s, mesh->face_right[f], mesh->face_left[f]);
    } else if (mesh->face_normal[f] < 0.0) {
      left_boundary = mesh->face_left[f];
    } else {
      right_boundary = mesh->face_left[f];
    }
  }
  if (periodic && left_boundary >= 0 && right_boundary >= 0) {
    append_unique_neighbor(s, left_boundary, right_boundary);
    append_unique_neighbor(s, right_boundary, left_boundary);
  }
  double pts[8], wts[8];
  const int nq = wo_gauss_legendre(p + 1 > 1 ? p + 1 : 1, pts, wts);
  const double period = mesh->x_right[ne - 1] - mesh->x_left[0];
  double sb[MAXM], tb[MAXM];
  for (int64_t e = 0; e < ne; ++e) {
    const double txl = mesh->x_left[e], txr = mesh->x_right[e];
    for (int k = 0; k < 2; ++k) {
      const int32_t nb = s->neighbors[e * 2 + k];
      if (nb < 0)
        continue;
      double sxl = mesh->x_left[nb], sxr = mesh->x_right[nb];
      const double offset =
          periodic_offset(line_centre(txl, txr) - line_centre(sxl, sxr), period);
      sxl += offset;
      sxr += offset;
      double *matrix = s->transforms + (e * 2 + k) * M * M;
      for (int q = 0; q < nq; ++q) {
        const double sxi = line_to_reference(sxl, sxr, line_to_physical(txl, txr, pts[q]));
        wo_legendre_basis(sxi, p, sb);
        wo_legendre_basis(pts[q], p, tb);
        for (int t = 0; t < M; ++t)
          for (int sm = 0; sm < M; ++sm)
            matrix[t * M + sm] += wts[q] * tb[t] * sb[sm];
      }
    }
  }
  s->check_point_count = nq + 2;
  s->check_basis = (double *)malloc(sizeof(double) * (size_t)(s->check_point_count * M));
  for (int q = 0; q < nq; ++q)
    wo_legendre_basis(pts[q], p, s->check_basis + q * M);
  wo_legendre_basis(-1.0, p, s->check_basis + nq * M);
  wo_legendre_basis(1.0, p, s->check_basis + (nq + 1) * M);
  return 0;
}

void wo_stencil_free(wo_stencil *s) {
  free(s->neighbors);
  free(s->transforms);
  free(s->normal_x);
  free(s->normal_y);
  free(s->check_basis);
  memset(s, 0, sizeof(*s));
}

/* ====================================================================== */
/* limiting                                                               */
/* ====================================================================== */

/* euler_characteristic.hpp:19-42 */
static void to_characteristic(double gamma, const double *average, const double *change,
                              double nx, double ny, double *out) {
  const prim_t mean = primitive(gamma, average);
  const double normal_velocity_ = mean.vx * nx + mean.vy * ny;
  const double tangent_velocity = -mean.vx * ny + mean.vy * nx;
  const double normal_momentum = change[1] * nx + change[2] * ny;
  const double tangent_momentum = -change[1] * ny + change[2] * nx;
  const double sound_speed_squared = gamma * mean.p / mean.rho;
  const double c = sqrt(sound_speed_squared);
  const double kinetic_energy =
      0.5 * (normal_velocity_ * normal_velocity_ + tangent_velocity * tangent_velocity);
  const double factor = (gamma - 1.0) / sound_speed_squared;
  const double acoustic_common =
      factor * (kinetic_energy * change[0] - normal_velocity_ * normal_momentum -
                tangent_velocity * tangent_momentum + change[3]);
  const double acoustic_difference = (normal_velocity_ * change[0] - normal_momentum) / c;
  out[0] = 0.5 * (acoustic_common + acoustic_difference);
  out[1] = change[0] - acoustic_common;
  out[2] = tangent_momentum - tangent_velocity * change[0];
  out[3] = 0.5 * (acoustic_common - acoustic_difference);
}

/* euler_characteristic.hpp:44-67 */
static void from_characteristic(double gamma, const double *average, const double *ch, double nx,
                                double ny, double *out) {
  const prim_t mean = primitive(gamma, average);
  const double normal_velocity_ = mean.vx * nx + mean.vy * ny;
  const double tangent_velocity = -mean.vx * ny + mean.vy * nx;
  const double c = sound_speed(gamma, &mean);
  const double enthalpy = (average[3] + mean.p) / average[0];
  const double kinetic_energy =
      0.5 * (normal_velocity_ * normal_velocity_ + tangent_velocity * tangent_velocity);
  const double density = ch[0] + ch[1] + ch[3];
  const double normal_momentum = (normal_velocity_ - c) * ch[0] + normal_velocity_ * ch[1] +
                                 (normal_velocity_ + c) * ch[3];
  const double tangent_momentum = tangent_velocity * density + ch[2];
  const double total_energy = (enthalpy - normal_velocity_ * c) * ch[0] +
                              kinetic_energy * ch[1] + tangent_velocity * ch[2] +
                              (enthalpy + normal_velocity_ * c) * ch[3];
  out[0] = density;
  out[1] = nx * normal_momentum - ny * tangent_momentum;
  out[2] = ny * normal_momentum + nx * tangent_momentum;
  out[3] = total_energy;
}

/* simple_weno.hpp:11-17 */
static double weno_smoothness(const double *c, int M) {
  double value = 0.0;
  for (int m = 1; m < M; ++m)
    value += c[m] * c[m];
  return value;
}

/* simple_weno.hpp:21-48 */
static void simple_weno(const double *target, const double *candidates, int count, int M,
                        double *limited) {
  const double epsilon = 1e-12;
  if (count == 0) {
    for (int m = 0; m < M; ++m)
      limited[m] = target[m];
    return;
  }
  double weights[8];
  const double target_denominator = epsilon + weno_smoothness(target, M);
  weights[0] = 0.5 / (target_denominator * target_denominator);
  double weight_sum = weights[0];
  const double neighbor_ideal_weight = 0.5 / (double)count;
  for (int k = 0; k < count; ++k) {
    const double denominator = epsilon + weno_smoothness(candidates + k * M, M);
    weights[k + 1] = neighbor_ideal_weight / (denominator * denominator);
    weight_sum += weights[k + 1];
  }
  limited[0] = target[0];
  for (int m = 1; m < M; ++m) {
    double value = weights[0] * target[m];
    for (int k = 0; k < count; ++k)
      value += weights[k + 1] * candidates[k * M + m];
    limited[m] = value / weight_sum;
  }
}

/* euler_characteristic_weno.hpp:17-67 */
void wo_characteristic_weno(double gamma, const double *average, double nx, double ny,
                            const double *target, const double *candidates, int count, int M,
                            double *limited) {
  double tc[4 * MAXM], cc[3 * 4 * MAXM], lc[4 * MAXM], wave_c[3 * MAXM];
  for (int k = -1; k < count; ++k) {
    const double *src = k < 0 ? target : candidates + k * 4 * M;
    double *dst = k < 0 ? tc : cc + k * 4 * M;
    for (int m = 0; m < M; ++m) {
      const double change[4] = {src[m], src[M + m], src[2 * M + m], src[3 * M + m]};
      double value[4];
      to_characteristic(gamma, average, change, nx, ny, value);
      for (int w = 0; w < 4; ++w)
        dst[w * M + m] = value[w];
    }
  }
  for (int w = 0; w < 4; ++w) {
    for (int k = 0; k < count; ++k)
      for (int m = 0; m < M; ++m)
        wave_c[k * M + m] = cc[k * 4 * M + w * M + m];
    simple_weno(tc + w * M, wave_c, count, M, lc + w * M);
  }
  for (int m = 0; m < M; ++m) {
    const double value[4] = {lc[m], lc[M + m], lc[2 * M + m], lc[3 * M + m]};
    double state[4];
    from_characteristic(gamma, average, value, nx, ny, state);
    for (int v = 0; v < 4; ++v)
      limited[v * M + m] = state[v];
  }
  for (int v = 0; v < 4; ++v)
    limited[v * M] = target[v * M];
}

/* euler_positivity.hpp:33-38 + modal_layout.hpp:26-36 with one element */
static void evaluate_modal(const double *c, int M, const double *basis, double *state) {
  for (int v = 0; v < 4; ++v) {
    double s = 0.0;
    for (int m = 0; m < M; ++m)
      s += c[v * M + m] * basis[m];
    state[v] = s;
  }
}

/* euler_positivity.hpp:48-53 */
static void scale_high_modes(double *c, int M, double scale) {
  for (int v = 0; v < 4; ++v)
    for (int m = 1; m < M; ++m)
      c[v * M + m] *= scale;
}

/* euler_positivity.hpp:44-58 */
static double pressure_preserving_theta(double gamma, const double *average, const double *point,
                                        double pressure_floor) {
  double lower = 0.0, upper = 1.0;
  for (int iteration = 0; iteration < 64; ++iteration) {
    const double middle = 0.5 * (lower + upper);
    double s[4];
    for (int v = 0; v < 4; ++v)
      s[v] = average[v] + middle * (point[v] - average[v]);
    if (primitive(gamma, s).p >= pressure_floor)
      lower = middle;
    else
      upper = middle;
  }
  return lower;
}

/* euler_positivity.hpp:63-102 */
int wo_positivity(double gamma, double *c, int M, const double *basis, int npts,
                  double density_floor, double pressure_floor, double *scale) {
  if (M == 0 || density_floor < 0.0 || pressure_floor < 0.0)
    return -2;
  const double inverse_sqrt2 = 1.0 / sqrt(2.0);
  const double average[4] = {c[0] * inverse_sqrt2, c[M] * inverse_sqrt2, c[2 * M] * inverse_sqrt2,
                             c[3 * M] * inverse_sqrt2};
  if (average[0] <= density_floor || primitive(gamma, average).p <= pressure_floor)
    return -1;
  double density_scale = 1.0;
  for (int pt = 0; pt < npts; ++pt) {
    double s[4];
    evaluate_modal(c, M, basis + pt * M, s);
    if (s[0] < density_floor)
      density_scale = std_min(density_scale, (average[0] - density_floor) / (average[0] - s[0]));
  }
  scale_high_modes(c, M, density_scale);
  double pressure_scale = 1.0;
  for (int pt = 0; pt < npts; ++pt) {
    double s[4];
    evaluate_modal(c, M, basis + pt * M, s);
    if (primitive(gamma, s).p >= pressure_floor)
      continue;
    pressure_scale =
        std_min(pressure_scale, pressure_preserving_theta(gamma, average, s, pressure_floor));
  }
  scale_high_modes(c, M, pressure_scale);
  if (scale)
    *scale = density_scale * pressure_scale;
  return 0;
}

/* euler_modal_limiter.cpp:18-24 + modal_decay.hpp:23-33 */
static int is_troubled(const wo_stencil *st, const double *source, int64_t e, double threshold) {
  double total = 0.0, highest = 0.0;
  const int64_t ne = st->element_count;
  for (int m = 0; m < st->mode_count; ++m) {
    const double value = source[(int64_t)m * ne + e];
    total += value * value;
    if (m >= st->highest_degree_begin)
      highest += value * value;
  }
  return !(total == 0.0 || highest / total <= threshold);
}

void wo_troubled_flags(const wo_stencil *st, double threshold, const double *c, uint8_t *flags) {
  for (int64_t e = 0; e < st->element_count; ++e)
    flags[e] = st->polynomial_order == 0 ? 0 : (uint8_t)is_troubled(st, c, e, threshold);
}

/* euler_modal_limiter.cpp:70-98 (gather :27-32, scatter :34-39, candidates :43-66) */
int wo_limit_euler(const wo_stencil *st, double gamma, double threshold, double density_floor,
                   double pressure_floor, double *c, uint8_t *flags, int64_t *bad_element) {
  const int64_t ne = st->element_count;
  if (flags)
    memset(flags, 0, (size_t)ne);
  if (st->polynomial_order == 0)
    return 0;
  const int M = st->mode_count;
  double *source = (double *)malloc(sizeof(double) * 4 * (size_t)M * (size_t)ne);
  memcpy(source, c, sizeof(double) * 4 * (size_t)M * (size_t)ne);
  double target[4 * MAXM], candidates[3 * 4 * MAXM], limited[4 * MAXM];
  int status = 0;
  for (int64_t e = 0; e < ne; ++e) {
    if (!is_troubled(st, source, e, threshold))
      continue;
    if (flags)
      flags[e] = 1;
    for (int v = 0; v < 4; ++v)
      for (int m = 0; m < M; ++m)
        target[v * M + m] = source[((int64_t)v * M + m) * ne + e];
    int count = 0;
    for (int k = 0; k < st->maximum_neighbors; ++k) {
      const int32_t nb = st->neighbors[e * st->maximum_neighbors + k];
      if (nb < 0)
        continue;
      const double *matrix = st->transforms + (e * st->maximum_neighbors + k) * M * M;
      for (int v = 0; v < 4; ++v) {
        double *result = candidates + (count * 4 + v) * M;
        for (int t = 0; t < M; ++t)
          result[t] = 0.0;
        for (int t = 0; t < M; ++t)
          for (int s = 0; s < M; ++s)
            result[t] += matrix[t * M + s] * source[((int64_t)v * M + s) * ne + nb];
        result[0] = target[v * M];
      }
      ++count;
    }
    const double average[4] = {target[0] / sqrt(2.0), target[M] / sqrt(2.0),
                               target[2 * M] / sqrt(2.0), target[3 * M] / sqrt(2.0)};
    wo_characteristic_weno(gamma, average, st->normal_x[e], st->normal_y[e], target, candidates,
                           count, M, limited);
    const int rc = wo_positivity(gamma, limited, M, st->check_basis, st->check_point_count,
                                 density_floor, pressure_floor, NULL);
    if (rc != 0) {
      if (bad_element)
        *bad_element = e;
      status = rc;
      break;
    }
    for (int v = 0; v < 4; ++v)
      for (int m = 0; m < M; ++m)
        c[((int64_t)v * M + m) * ne + e] = limited[v * M + m];
  }
  free(source);
  return status;
}

/* ====================================================================== */
/* time step                                                              */
/* ====================================================================== */

/* cfl_timestep.cpp:22-30 */
double wo_tri_minimum_altitude(const wo_tri_mesh *mesh) {
  double result = DBL_MAX;
  for (int64_t e = 0; e < mesh->element_count; ++e) {
    const tri_map m = element_map(mesh, e);
    const double l0 = map_edge_length(&m, 0), l1 = map_edge_length(&m, 1),
                 l2 = map_edge_length(&m, 2);
    /* std::max({l0, l1, l2}): the first largest */
    double longest = l0;
    if (longest < l1)
      longest = l1;
    if (longest < l2)
      longest = l2;
    result = std_min(result, 4.0 * map_jacobian_determinant(&m) / longest);
  }
  return result;
}

/* cfl_timestep.cpp:33-47 */
static int euler_maximum_speed(double gamma, const double *c, int64_t ne, int M, int dimensions,
                               double *speed) {
  double result = 0.0;
  const double scale = 1.0 / sqrt(2.0);
  for (int64_t e = 0; e < ne; ++e) {
    const double s[4] = {scale * c[(int64_t)0 * M * ne + e], scale * c[(int64_t)1 * M * ne + e],
                         scale * c[(int64_t)2 * M * ne + e], scale * c[(int64_t)3 * M * ne + e]};
    if (!(s[0] > 0.0 && primitive(gamma, s).p > 0.0))
      return -1;
    const prim_t v = primitive(gamma, s);
    const double velocity = dimensions == 1 ? fabs(v.vx) : hypot(v.vx, v.vy);
    result = std_max(result, velocity + sound_speed(gamma, &v));
  }
  *speed = result;
  return 0;
}

/* cfl_timestep.cpp:49-51 */
static double euler_limit(double length, double speed, int p, double cfl) {
  return speed > 0.0 ? cfl * length / (speed * (2 * p + 1)) : 0.0;
}

/* cfl_timestep.cpp:78-84 */
int wo_euler_tri_cfl(const wo_tri_mesh *mesh, double gamma, const double *c, int p, double cfl,
                     double *dt) {
  double speed = 0.0;
  if (euler_maximum_speed(gamma, c, mesh->element_count, wo_tri_modes(p), 2, &speed) != 0)
    return -1;
  *dt = euler_limit(wo_tri_minimum_altitude(mesh), speed, p, cfl);
  return 0;
}

/* cfl_timestep.cpp:14-19 */
static double minimum_length(const wo_line_mesh *mesh) {
  double result = DBL_MAX;
  for (int64_t e = 0; e < mesh->element_count; ++e)
    result = std_min(result, mesh->x_right[e] - mesh->x_left[e]);
  return result;
}

/* cfl_timestep.cpp:70-76 */
int wo_euler_line_cfl(const wo_line_mesh *mesh, double gamma, const double *c, int p, double cfl,
                      double *dt) {
  double speed = 0.0;
  if (euler_maximum_speed(gamma, c, mesh->element_count, wo_line_modes(p), 1, &speed) != 0)
    return -1;
  *dt = euler_limit(minimum_length(mesh), speed, p, cfl);
  return 0;
}

/* cfl_timestep.cpp:55-60 */
double wo_line_advection_cfl(const wo_line_mesh *mesh, double a, int p, double cfl) {
  if (mesh->element_count == 0 || a == 0.0)
    return 0.0;
  return cfl * minimum_length(mesh) / (fabs(a) * (2.0 * p + 1.0));
}

/* cfl_timestep.cpp:62-68 */
double wo_tri_scalar_cfl(const wo_tri_mesh *mesh, double vx, double vy, int p, double cfl) {
  const double speed = hypot(vx, vy);
  if (mesh->element_count == 0 || speed == 0.0)
    return 0.0;
  return cfl * wo_tri_minimum_altitude(mesh) / (speed * (2.0 * p + 1.0));
}

/* ====================================================================== */
/* SSP-RK3 (cpp/include/wasl/time/ssp_rk3.hpp:37-61)                      */
/* ====================================================================== */

typedef struct {
  const wo_tri_mesh *mesh;
  const wo_euler_tri_setup *setup;
  double gamma;
  int p;
  double *exterior;
} tri_ctx;

static void tri_residual(tri_ctx *x, const double *stage, double *rhs) {
  if (x->setup->boundary_kind == 3)
    wo_transmissive_tri_euler_exterior(x->mesh, x->p, stage, x->exterior);
  else
    wo_periodic_tri_euler_exterior(x->mesh, x->p, x->setup->donors, x->setup->donor_basis, stage,
                                   x->exterior);
  wo_euler_tri_residual(x->mesh, x->gamma, x->p, stage, x->exterior, rhs);
}

static int tri_post_stage(tri_ctx *x, double *state, uint8_t *flags) {
  const wo_euler_tri_setup *s = x->setup;
  if (!s->stencil)
    return 0;
  return wo_limit_euler(s->stencil, x->gamma, s->threshold, s->density_floor, s->pressure_floor,
                        state, flags, NULL);
}

int wo_euler_tri_step(const wo_tri_mesh *mesh, const wo_euler_tri_setup *setup, double gamma,
                      int p, double dt, double *c, uint8_t *flags) {
  const int M = wo_tri_modes(p);
  const size_t n = 4 * (size_t)M * (size_t)mesh->element_count;
  double *rhs = (double *)malloc(sizeof(double) * n);
  double *euler = (double *)malloc(sizeof(double) * n);
  double *stage = (double *)malloc(sizeof(double) * n);
  tri_ctx x = {mesh, setup, gamma, p,
               (double *)malloc(sizeof(double) * 4 * (size_t)(mesh->face_count * (p + 1)))};
  const int64_t ne = mesh->element_count;
  int rc = 0;
  tri_residual(&x, c, rhs);
  for (size_t i = 0; i < n; ++i)
    euler[i] = c[i] + dt * rhs[i];
  if ((rc = tri_post_stage(&x, euler, flags)) != 0)
    goto done;
  tri_residual(&x, euler, rhs);
  for (size_t i = 0; i < n; ++i)
    stage[i] = 0.75 * c[i] + 0.25 * (euler[i] + dt * rhs[i]);
  if ((rc = tri_post_stage(&x, stage, flags ? flags + ne : NULL)) != 0)
    goto done;
  tri_residual(&x, stage, rhs);
  for (size_t i = 0; i < n; ++i)
    c[i] = (1.0 / 3.0) * c[i] + (2.0 / 3.0) * (stage[i] + dt * rhs[i]);
  rc = tri_post_stage(&x, c, flags ? flags + 2 * ne : NULL);
done:
  free(rhs);
  free(euler);
  free(stage);
  free(x.exterior);
  return rc;
}

int wo_euler_line_step(const wo_line_mesh *mesh, int left_kind, int right_kind,
                       const wo_stencil *stencil, double threshold, double density_floor,
                       double pressure_floor, double gamma, int p, double dt, double *c,
                       uint8_t *flags) {
  const int M = wo_line_modes(p);
  const size_t n = 4 * (size_t)M * (size_t)mesh->element_count;
  double *rhs = (double *)malloc(sizeof(double) * n);
  double *euler = (double *)malloc(sizeof(double) * n);
  double *stage = (double *)malloc(sizeof(double) * n);
  double *ext = (double *)malloc(sizeof(double) * 4 * (size_t)mesh->face_count);
  int rc = 0;
  double *states[3] = {euler, stage, c};
  for (int k = 0; k < 3; ++k) {
    const double *in = k == 0 ? c : states[k - 1];
    if ((rc = wo_line_euler_exterior(mesh, p, left_kind, right_kind, in, ext)) != 0)
      break;
    wo_euler_line_residual(mesh, gamma, p, in, ext, rhs);
    if (k == 0)
      for (size_t i = 0; i < n; ++i)
        euler[i] = c[i] + dt * rhs[i];
    else if (k == 1)
      for (size_t i = 0; i < n; ++i)
        stage[i] = 0.75 * c[i] + 0.25 * (euler[i] + dt * rhs[i]);
    else
      for (size_t i = 0; i < n; ++i)
        c[i] = (1.0 / 3.0) * c[i] + (2.0 / 3.0) * (stage[i] + dt * rhs[i]);
    if (stencil &&
        (rc = wo_limit_euler(stencil, gamma, threshold, density_floor, pressure_floor, states[k],
                             flags ? flags + k * mesh->element_count : NULL, NULL)) != 0)
      break;
  }
  free(rhs);
  free(euler);
  free(stage);
  free(ext);
  return rc;
}

/* line_advection_step.hpp:16-25 */
void wo_scalar_line_step(const wo_line_mesh *mesh, int left_kind, double left_value,
                         int right_kind, double right_value, double a, int p, double dt,
                         double *c) {
  const size_t n = (size_t)(p + 1) * (size_t)mesh->element_count;
  double *rhs = (double *)malloc(sizeof(double) * n);
  double *euler = (double *)malloc(sizeof(double) * n);
  double *stage = (double *)malloc(sizeof(double) * n);
  double *ext = (double *)malloc(sizeof(double) * (size_t)mesh->face_count);
  const double *ins[3] = {c, euler, stage};
  for (int k = 0; k < 3; ++k) {
    wo_line_scalar_exterior(mesh, p, left_kind, left_value, right_kind, right_value, ins[k], ext);
    wo_scalar_line_residual(mesh, a, p, ins[k], ext, rhs);
    if (k == 0)
      for (size_t i = 0; i < n; ++i)
        euler[i] = c[i] + dt * rhs[i];
    else if (k == 1)
      for (size_t i = 0; i < n; ++i)
        stage[i] = 0.75 * c[i] + 0.25 * (euler[i] + dt * rhs[i]);
    else
      for (size_t i = 0; i < n; ++i)
        c[i] = (1.0 / 3.0) * c[i] + (2.0 / 3.0) * (stage[i] + dt * rhs[i]);
  }
  free(rhs);
  free(euler);
  free(stage);
  free(ext);
}

void wo_scalar_tri_step(const wo_tri_mesh *mesh, const int32_t *donors, const double *donor_basis,
                        double vx, double vy, int p, double dt, double *c) {
  const size_t n = (size_t)wo_tri_modes(p) * (size_t)mesh->element_count;
  double *rhs = (double *)malloc(sizeof(double) * n);
  double *euler = (double *)malloc(sizeof(double) * n);
  double *stage = (double *)malloc(sizeof(double) * n);
  double *ext = (double *)malloc(sizeof(double) * (size_t)(mesh->face_count * (p + 1)));
  const double *ins[3] = {c, euler, stage};
  for (int k = 0; k < 3; ++k) {
    wo_periodic_tri_scalar_exterior(mesh, p, donors, donor_basis, ins[k], ext);
    wo_scalar_tri_residual(mesh, vx, vy, p, ins[k], ext, rhs);
    if (k == 0)
      for (size_t i = 0; i < n; ++i)
        euler[i] = c[i] + dt * rhs[i];
    else if (k == 1)
      for (size_t i = 0; i < n; ++i)
        stage[i] = 0.75 * c[i] + 0.25 * (euler[i] + dt * rhs[i]);
    else
      for (size_t i = 0; i < n; ++i)
        c[i] = (1.0 / 3.0) * c[i] + (2.0 / 3.0) * (stage[i] + dt * rhs[i]);
  }
  free(rhs);
  free(euler);
  free(stage);
  free(ext);
}

/* ====================================================================== */
/* projection and diagnostics                                             */
/* ====================================================================== */

void wo_tri_rule_points(const wo_tri_mesh *mesh, int rule_order, double *x, double *y) {
  double qxi[MAXQ], qeta[MAXQ], qw[MAXQ];
  const int Q = wo_tri_volume_rule(rule_order, qxi, qeta, qw);
  for (int64_t e = 0; e < mesh->element_count; ++e) {
    const tri_map m = element_map(mesh, e);
    for (int q = 0; q < Q; ++q)
      map_reference_to_physical(&m, qxi[q], qeta[q], x + e * Q + q, y + e * Q + q);
  }
}

/* l2_projection.hpp:57-76 with accumulate_projection :23-30 */
void wo_tri_project(const wo_tri_mesh *mesh, int p, int rule_order, int nv, const double *values,
                    double *c) {
  const int M = wo_tri_modes(p);
  const int64_t ne = mesh->element_count;
  double qxi[MAXQ], qeta[MAXQ], qw[MAXQ], b[MAXM];
  const int Q = wo_tri_volume_rule(rule_order, qxi, qeta, qw);
  /* The basis at the rule's points is the same on every element; each
     coefficient still sums its terms over q in order from 0.0. */
  double *basis = (double *)malloc(sizeof(double) * (size_t)Q * (size_t)M);
  double *acc = (double *)malloc(sizeof(double) * (size_t)nv * (size_t)M);
  for (int q = 0; q < Q; ++q) {
    wo_dubiner_basis(qxi[q], qeta[q], p, b);
    memcpy(basis + (size_t)q * M, b, sizeof(double) * (size_t)M);
  }
  for (int64_t e = 0; e < ne; ++e) {
    memset(acc, 0, sizeof(double) * (size_t)nv * (size_t)M);
    for (int q = 0; q < Q; ++q) {
      const double *val = values + (e * Q + q) * nv;
      for (int v = 0; v < nv; ++v)
        for (int m = 0; m < M; ++m)
          acc[v * M + m] += qw[q] * val[v] * basis[q * M + m];
    }
    for (int v = 0; v < nv; ++v)
      for (int m = 0; m < M; ++m)
        c[((int64_t)v * M + m) * ne + e] = acc[v * M + m];
  }
  free(basis);
  free(acc);
}

void wo_line_rule_points(const wo_line_mesh *mesh, int point_count, double *x) {
  double pts[8], wts[8];
  const int Q = wo_gauss_legendre(point_count, pts, wts);
  for (int64_t e = 0; e < mesh->element_count; ++e)
    for (int q = 0; q < Q; ++q)
      x[e * Q + q] = line_to_physical(mesh->x_left[e], mesh->x_right[e], pts[q]);
}

/* l2_projection.hpp:36-53 */
void wo_line_project(const wo_line_mesh *mesh, int p, int point_count, int nv,
                     const double *values, double *c) {
  const int M = wo_line_modes(p);
  const int64_t ne = mesh->element_count;
  double pts[8], wts[8], b[MAXM];
  const int Q = wo_gauss_legendre(point_count, pts, wts);
  memset(c, 0, sizeof(double) * (size_t)nv * (size_t)M * (size_t)ne);
  for (int64_t e = 0; e < ne; ++e)
    for (int q = 0; q < Q; ++q) {
      wo_legendre_basis(pts[q], p, b);
      const double *val = values + (e * Q + q) * nv;
      for (int v = 0; v < nv; ++v)
        for (int m = 0; m < M; ++m)
          c[((int64_t)v * M + m) * ne + e] += wts[q] * val[v] * b[m];
    }
}

/* euler_diagnostics.cpp:33-39 / scalar_diagnostics.cpp:29-36 */
double wo_tri_mass(const wo_tri_mesh *mesh, const double *mode0, int64_t stride) {
  double result = 0.0;
  for (int64_t e = 0; e < mesh->element_count; ++e) {
    const tri_map m = element_map(mesh, e);
    result += sqrt(2.0) * map_jacobian_determinant(&m) * mode0[e * stride];
  }
  return result;
}

/* euler_diagnostics.cpp:26-31 / scalar_diagnostics.cpp:21-27 */
double wo_line_mass(const wo_line_mesh *mesh, const double *mode0, int64_t stride) {
  double result = 0.0;
  for (int64_t e = 0; e < mesh->element_count; ++e)
    result += sqrt(2.0) * line_jacobian(mesh->x_left[e], mesh->x_right[e]) * mode0[e * stride];
  return result;
}
