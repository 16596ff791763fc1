// Launch interface of the CUDA kernels (host side; no device code here).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace wasl_b200 {

// Device view of a triangle mesh, structure of arrays over elements.
//   geo       [5][ne]    ax, ay, bx, by (columns of the affine map), 1/det(J)
//   slot_*    [3][ne]    the element's three faces in ascending global face
//                        index (the reference's flux summation order):
//     slot_nbr   the other element, or -(b+1) for boundary face b
//     slot_code  bit 0: this element is the face's left side; bits 1-2 left
//                local edge; bits 3-4 right local edge; bit 5 orientation flip
//     slot_geo   [3][3][ne] face normal x, normal y (left to right), edge scale
//   donor       [nb][QF] periodic donor element of each boundary edge point
//   donor_basis [nb][QF][M] donor basis at the periodic image
struct TriMeshView {
  std::int64_t ne = 0;
  const double *geo = nullptr;
  const std::int32_t *slot_nbr = nullptr;
  const std::uint8_t *slot_code = nullptr;
  const double *slot_geo = nullptr;
  const std::int32_t *donor = nullptr;
  const double *donor_basis = nullptr;
  int boundary = 0; // 0 periodic, 3 transmissive (the owner's own trace)
};

// Boundary faces in boundary index order (the slots' -(b+1) numbering):
// owning element, its local edge, normal [2][count], and a scratch value
// buffer [4][count] (the mixed form's FP64 mode-0 face values).
struct BoundaryView {
  std::int64_t count = 0;
  const std::int32_t *element = nullptr;
  const std::uint8_t *local_edge = nullptr;
  const double *normal = nullptr;
  double *value = nullptr;
  // Periodic faces paired across the period (the mixed form evaluates each
  // pair once): the FP32 donor basis [count][QF][M] at the canonical face's
  // points, used by the element on the far side as its own basis.
  int paired = 0;
  const float *basis32 = nullptr;
};

// Faces in global face order for the face-centric mixed kernels: left and
// right element (-(b+1) for boundary face b), code (bits as slot_code),
// normal [2][count], per-face record scratch, and each element's face index
// per slot [3][ne].
struct FaceView {
  std::int64_t count = 0;
  const std::int32_t *left = nullptr;
  const std::int32_t *right = nullptr;
  const std::uint8_t *code = nullptr;
  const double *normal = nullptr;
  void *record = nullptr;
  const std::int32_t *slot_face = nullptr;
};

// Element-centric slots of the fused tile kernel, [3][ne] each, in the
// element's face order: the element across the face (-1 on a transmissive
// boundary face, whose exterior is the element's own trace), a code byte as
// slot_code (bit 0 this element is the face's left side, bits 1-2 left local
// edge, bits 3-4 right local edge, bit 5 orientation flip) plus bit 6 "this
// element's basis on the face is the periodic table row aux" and bit 7 "the
// other element's basis is the periodic table row aux", and aux (the row of
// BoundaryView::basis32 for paired periodic faces).  The normal and edge
// scale of the face are slot_geo's.
struct TileSlots {
  const std::int32_t *nbr = nullptr;
  const std::uint8_t *code = nullptr;
  const std::int32_t *aux = nullptr;
};

// Per-local-edge arrays of the patch kernel, [3][ne] each (geo [3][3][ne]):
// the element across local edge j (-1 on a transmissive boundary), an info
// byte (bit 0 this element is the face's left side, bits 1-2 the neighbour's
// local edge, bit 3 the neighbour's points run in the opposite order), and the
// face's normal (left to right) and scale.
struct PatchEdges {
  const std::int32_t *nbr = nullptr;
  const std::uint8_t *info = nullptr;
  const double *geo = nullptr;
};

// One entry of a tile work list: elements [first, first + count) of one case
// (count <= the kernel's tile size), and the case whose dt applies.
struct TileWork {
  std::int32_t first = 0, count = 0, case_id = 0, pad = 0;
};

// One SSP-RK3 stage: residual of `in`, then
//   stage 0: out = in + dt r
//   stage 1: out = 0.75 u0 + 0.25 (in + dt r)
//   stage 2: out = (1/3) u0 + (2/3) (in + dt r)
// (cpp/include/wasl/time/ssp_rk3.hpp:44-60).  With sense != 0 the kernel also
// evaluates the modal-decay sensor on `out` and appends troubled elements.
struct StageArgs {
  TriMeshView mesh;
  BoundaryView boundary;
  FaceView faces;
  const void *face_table = nullptr;   // FaceTable<P, real> in device memory
  const void *face_table64 = nullptr; // FaceTable<P, double> (the mixed form's FP64 boundary terms)
  const double *in = nullptr;
  const double *u0 = nullptr;
  double *out = nullptr;
  const double *dt = nullptr; // device scalar, or null: dt_value
  double dt_value = 0.0;
  double gamma = 1.4;
  double velocity_x = 0.0, velocity_y = 0.0; // scalar advection velocity
  int stage = 0;
  int sense = 0;
  double threshold = 1e-3;
  int highest_degree_begin = 0;
  std::uint8_t *flags = nullptr;       // [ne]
  std::int32_t *troubled = nullptr;    // [ne] compacted list
  std::int32_t *troubled_count = nullptr;
  // Fused tile kernel: slots, and an optional work list (null: tile b covers
  // elements [b T, b T + T)) with per-case time steps (null: dt / dt_value).
  TileSlots tile;
  PatchEdges patch;
  const TileWork *work = nullptr;
  std::int64_t work_count = 0;
  const double *case_dt = nullptr;
  // Tile kernel, last stage: the largest cell-average wave speed |u| + c of
  // `out` (the CFL kernels' formula) is max-reduced into speed_max[case] as
  // FP64 bits, and a non-physical average sets the error word.
  unsigned long long *speed_max = nullptr;
  unsigned long long *error = nullptr;
  // Tile kernel: elements with a face across which the cell means jump go to
  // the rough list [ne] (count rough_count) and are computed by the second
  // pass with FP64 faces; null: one FP32 pass.  element_case [ne] gives the
  // case (for case_dt) of a rough element; null: case 0.
  std::int32_t *rough = nullptr;
  std::int32_t *rough_count = nullptr;
  const std::int32_t *element_case = nullptr;
};

// Limiter over the compacted troubled list (cpp/src/limiting/euler_modal_limiter.cpp:70-98).
struct LimitArgs {
  std::int64_t ne = 0;
  double *state = nullptr;              // U[var][mode][elem], unlimited on entry
  const std::int32_t *troubled = nullptr;
  const std::int32_t *troubled_count = nullptr;
  const std::int32_t *neighbors = nullptr;   // [ne][NB]
  const double *transforms = nullptr;        // [ne][NB][M][M]
  const double *normal_x = nullptr, *normal_y = nullptr;
  const double *check_basis = nullptr;       // [points][M]
  int check_points = 0;
  double gamma = 1.4, density_floor = 1e-10, pressure_floor = 1e-10;
  double *limited = nullptr;                 // [ne][4][M] scratch, by list position
  unsigned long long *error = nullptr;
  // Always-on positivity (not the reference's behaviour): after the troubled
  // cells, the positivity limiter also runs on every element with flags[e]
  // == 0.  The launch then counts three kernels instead of two.
  int positivity_all = 0;
  const std::uint8_t *flags = nullptr;
  // > 0: the check-point floors become max(floor, relative_floor x mean
  // density) and max(floor, relative_floor x mean energy) (the mixed form).
  double relative_floor = 0.0;
  // Batched solves: a mean below a floor is recorded as case_status[case of
  // e] (first error only) instead of in the error word.
  int *case_status = nullptr;
  const std::int32_t *element_case = nullptr;
  // [M] largest |basis value| of each mode over the check points: lets the
  // always-on pass skip elements whose bounds clear the floors (null: none).
  const double *check_bound = nullptr;
};

// check_bound[m] = max over points |check_basis[point][m]| (host).
std::vector<double> positivity_check_bound(const std::vector<double> &check_basis, int M);

// The mixed form's positivity check-point floors relative to the mean: FP32
// resolves a point state to ~6e-8 of the mean, so point densities and
// pressures are kept at least 1e-5 of the mean density and energy.
constexpr double kMixedRelativeFloor = 1e-5;

// Modal-decay sensor on the density modes of `state` (modal_decay.hpp:23-33).
struct SenseArgs {
  std::int64_t ne = 0;
  const double *state = nullptr;
  double threshold = 1e-3;
  int highest_degree_begin = 0;
  std::uint8_t *flags = nullptr;
  std::int32_t *troubled = nullptr;
  std::int32_t *troubled_count = nullptr;
};

// Largest cell-average wave speed |u| + c (cpp/src/time/cfl_timestep.cpp:33-47).
// result[0] = speed bits (max), result[1] = ~(smallest element index reaching
// it), result[2..5] = that element's mode-0 coefficients, then dt in result[6]
// computed on the device as cfl h / (speed (2p+1)).  result[8] counts the
// blocks that have finished and result[16..) holds each block's (speed,
// element) pair: the buffer has kCflResultWords words.
constexpr int kCflBlocks = 148 * 4;
constexpr std::size_t kCflResultWords = 16 + 2 * kCflBlocks;
struct CflArgs {
  std::int64_t ne = 0;
  int M = 1;
  int dimensions = 2;
  const double *state = nullptr;
  double gamma = 1.4;
  double cfl = 0.1;
  double length = 0.0; // minimum altitude (2D) or length (1D)
  int p = 0;
  unsigned long long *result = nullptr; // kCflResultWords words
  double *dt = nullptr;                 // device dt written by the final kernel
  unsigned long long *error = nullptr;
  // Storage order (storage column -> caller's element), or null: ties of the
  // largest speed go to the smallest caller's index either way.
  const std::int32_t *order = nullptr;
};

// Reference-line tables of the 1D kernels: orthonormal Legendre modes and
// their derivatives at the Gauss points of the residual's rule (p+1 points
// for Euler, line_residual.hpp:29; max(1, p) for scalar advection,
// scalar_advection/line_residual.hpp:40-42), the weights, and the modes at
// the ends xi = -1 (lb) and xi = +1 (rb).  Passed by value.
struct LineTable {
  static constexpr int kMaxPoints = 8, kMaxModes = 8;
  double phi[kMaxPoints][kMaxModes];
  double dphi[kMaxPoints][kMaxModes];
  double w[kMaxPoints];
  double lb[kMaxModes], rb[kMaxModes];
};

// One SSP-RK3 stage on a line mesh (elements sorted left to right: element e
// has face e on its left and face e+1 on its right).  State [variable][mode]
// [element] with 4 Euler variables or 1 scalar.  End kinds as enum
// wasl_boundary (periodic, inflow (scalar only), outflow).
struct LineStageArgs {
  std::int64_t ne = 0;
  const double *inv_jacobian = nullptr; // [ne] 1 / ((x_right - x_left) / 2)
  const double *in = nullptr;
  const double *u0 = nullptr;
  double *out = nullptr;
  const double *dt = nullptr; // device scalar, or null: dt_value
  double dt_value = 0.0;
  double gamma = 1.4;
  double speed = 0.0;         // scalar wavespeed
  int left_kind = 0, right_kind = 0;
  double left_value = 0.0, right_value = 0.0;
  int stage = 0;
  int sense = 0;
  double threshold = 1e-3;
  int highest_degree_begin = 0;
  std::uint8_t *flags = nullptr;
  std::int32_t *troubled = nullptr;
  std::int32_t *troubled_count = nullptr;
  LineTable table;
};

// A whole serial run of a line mesh in one launch of one CTA (the state's
// three buffers in its shared memory): see line_run_f64.  result[0] steps,
// result[1] final time (FP64 bits), result[2] status (0 done, 1 the time step
// cannot advance time, 2 a non-physical cell average, also in *error).
struct LineRunArgs {
  LineStageArgs stage; // mesh, table, ends, physics (in/out/u0/dt unused)
  double *state = nullptr;
  double fixed_dt = 0.0; // > 0: this step (scalar advection); 0: CFL per step
  double cfl = 0.0, length = 0.0;
  double start_time = 0.0, end_time = 0.0;
  unsigned long long max_steps = 0;
  unsigned long long *result = nullptr; // 3 words
  unsigned long long *error = nullptr;
};
constexpr std::size_t kLineRunMaxBytes = 200 * 1024;
std::size_t line_run_bytes(int variables, int p, std::int64_t ne);
void launch_line_run_f64(int variables, int p, const LineRunArgs &r, cudaStream_t stream);

bool line_order_supported(int p); // 0..6
void fill_line_table(int p, int points, LineTable &table);
void launch_line_stage_f64(int variables, int p, const LineStageArgs &a, cudaStream_t stream);

// 2D scalar advection (constant velocity a.velocity_x/y) on the triangle
// slots of StageArgs; state [mode][element].
void upload_scalar_tri_tables(int p);
void launch_scalar_tri_stage_f64(int p, const StageArgs &a, cudaStream_t stream);

bool euler_tri_order_supported(int p);
void upload_euler_tri_tables_f64(int p);
std::size_t euler_tri_face_table_bytes(int p, bool fp32);
void fill_euler_tri_face_table(int p, bool fp32, void *host_buffer);
void launch_euler_tri_stage_f64(int p, const StageArgs &a, cudaStream_t stream);
// The mixed form's volume rule: the collapsed rule of order `rule` (p..p+2;
// 0 means p+2, the reference residual's rule), or kSymmetricVolumeRule: the
// fully symmetric rule of degree 2p (3, 6, 12 points at P1-P3), as exact as
// the collapsed order-p rule with fewer points.
constexpr int kSymmetricVolumeRule = -1;
bool euler_tri_mixed_supported(int p, int rule);
void upload_euler_tri_tables_mixed(int p, int rule);
std::size_t euler_tri_mixed_face_record_bytes(int p);
void launch_euler_tri_stage_mixed(int p, int rule, const StageArgs &a, cudaStream_t stream);
// The fused tile form of the mixed stage: one kernel per stage.  `shape`
// (0 .. euler_tri_tile_shapes()-1) picks elements per CTA and the register
// budget; with a work list there is one CTA per entry (count <= the shape's
// elements), else ceil(ne / elements) CTAs.  Requires transmissive
// boundaries or paired periodic faces.
// Largest cell-average wave speed per case over a tile work list (blocks of
// 128 threads; tiles of any size), max-reduced into speed[case].
void launch_batch_speed(const double *state, std::int64_t ne, int M, double gamma,
                        const TileWork *work, std::int64_t work_count, unsigned long long *speed,
                        unsigned long long *error, int *status, cudaStream_t stream);
// Number of launch shapes of the tile kernels (euler_tri_tile_shapes()
// returns it; per-shape host arrays are sized by it).
constexpr int kTileShapeCount = 16;
int euler_tri_tile_shapes();
int euler_tri_tile_elements(int shape);
// Shapes of the patch kernel (StageArgs::patch; no rough pass, so runs
// without the limiter only).
bool euler_tri_tile_is_patch(int shape);
// Shapes that run with the limiter (all but the patch kernel with its volume
// term on the tensor cores).
bool euler_tri_tile_limits(int shape);

void launch_euler_tri_stage_tile(int p, int rule, int shape, const StageArgs &a,
                                 cudaStream_t stream);
// Sets the tile kernels' launch attributes on the current device (call
// before capturing launches in a graph).
void prepare_euler_tri_stage_tile(int p, int rule);
void launch_limit_f64(int M, int NB, const LimitArgs &a, cudaStream_t stream);
void launch_sense_f64(int M, const SenseArgs &a, cudaStream_t stream);
// One kernel: the speed, the arg-max and dt (result[0..6], and *a.dt).
void launch_cfl(const CflArgs &a, cudaStream_t stream);
// The largest cell-average wave speed alone (a.result[0], zeroed first; no
// arg-max and no dt): for device-resident steps, whose dt comes from it by
// launch_dt_from_speed with the same arithmetic as launch_cfl's dt.
void launch_cfl_speed(const CflArgs &a, cudaStream_t stream);
// dt[c] = cfl length[c] / (speed (2 p[c] + 1)) from reduced speeds (0 where
// the speed is 0 or status[c] is non-zero), added to elapsed[c] when elapsed
// is not null; then the speed words are zeroed.  length/p are per-case
// arrays, or null for the shared length_all/p_all; status may be null.
void launch_dt_from_speed(std::int64_t cases, unsigned long long *speed, double cfl,
                          const double *length, const int *p, double length_all, int p_all,
                          double *dt, double *elapsed, const int *status, cudaStream_t stream,
                          bool dependent = false); // as a programmatic dependent launch

} // namespace wasl_b200
