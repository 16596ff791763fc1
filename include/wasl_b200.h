/*
 * wasl_b200.h -- C-ABI of the B200 modal RKDG solver (libwasl_b200.so).
 *
 * A step-level handle that is a drop-in for the reference's serial CPU solver
 * of scalar advection and compressible Euler on 1D line and 2D triangle
 * meshes.  Plain C types only: pointers, sizes, int status codes.  Every call
 * returns 0 on success or a negative status; wasl_gpu_last_error() gives the
 * message, worded like the exception the reference throws for the same
 * failure.  Host arrays are copied in and out; the handle owns all device
 * memory and one CUDA stream.  A handle is not thread-safe.
 *
 * Reference interfaces each entry point replaces (paths inside indrow/wasl):
 *   SerialCaseModel                cpp/include/wasl/case/serial_case_runner.hpp:22-34
 *     initial_state / from_checkpoint     -> wasl_gpu_set_state
 *     to_checkpoint / cell_averages       -> wasl_gpu_get_state
 *     stable_time_step                    -> wasl_gpu_stable_dt
 *     advance (ssp_rk3_step)              -> wasl_gpu_step
 *     mass                                -> wasl_gpu_mass_energy
 *   run_serial_case loop           cpp/src/case/serial_case_runner.cpp:117-149 -> wasl_gpu_run
 *   write_checkpoint/read_checkpoint cpp/include/wasl/io/checkpoint_file.hpp:9-11
 *                                                -> wasl_gpu_write_checkpoint / _read_checkpoint
 *   case setup (mesh, stencil, periodic trace)   cpp/src/case/euler_triangle.cpp:16-25,
 *                                                cpp/src/case/euler_line.cpp:14-22,
 *                                                cpp/src/case/scalar_advection_line.cpp:11-19,
 *                                                cpp/src/case/scalar_advection_triangle.cpp:16-30
 *                                                -> wasl_gpu_create
 *
 * Solvers behind one handle (wasl_gpu_form_supported tells which forms exist):
 *   2D Euler, triangles P0-P3: plain FP64 (bit-identical) and the mixed form (P1-P3);
 *   2D scalar advection, triangles P0-P3, periodic: plain FP64;
 *   1D Euler and 1D scalar advection, lines P0-P6: plain FP64.
 * Line elements are stored in the reference's order (sorted by left end);
 * triangles keep the caller's order.  Scalar states use the checkpoint layout
 * [mode][element] (cpp/src/case/scalar_coefficient_layout.cpp transposes the
 * reference's solver layout [element][mode] into it).
 */
#ifndef WASL_B200_H
#define WASL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct wasl_gpu wasl_gpu;

enum wasl_equation { WASL_SCALAR_ADVECTION = 0, WASL_EULER = 1 };
/* Boundary kinds; values match the bridge's u8 kinds (crates/wasl-bridge/src/ops.rs). */
enum wasl_boundary { WASL_PERIODIC = 0, WASL_INFLOW = 1, WASL_OUTFLOW = 2, WASL_TRANSMISSIVE = 3 };
enum wasl_precision { WASL_PLAIN_FP64 = 0, WASL_MIXED = 1 };
enum wasl_status {
  WASL_OK = 0,
  WASL_ERR_ARGUMENT = -1,     /* invalid argument (std::invalid_argument) */
  WASL_ERR_RUNTIME = -2,      /* simulation failure (std::runtime_error) */
  WASL_ERR_CUDA = -3,         /* CUDA error, or no usable device */
  WASL_ERR_NONPHYSICAL = -4,  /* a cell average is not physical (cfl_timestep.cpp:39-40) */
  WASL_ERR_FLOOR = -5         /* positivity: average below a floor (euler_positivity.hpp:74-75) */
};

typedef struct {
  int dimensions;            /* 1 line mesh, 2 triangle mesh */
  int equation;              /* enum wasl_equation */
  int polynomial_order;      /* lines 0..6, triangles 0..3 */
  double heat_capacity_ratio;
  double velocity_x;         /* scalar advection: wavespeed (1D) / velocity (2D) */
  double velocity_y;
  int boundary_left;         /* 1D: left end kind; 2D: every boundary (periodic/transmissive) */
  int boundary_right;        /* 1D: right end kind (transmissive on a line is outflow) */
  double inflow_left;        /* 1D scalar inflow values */
  double inflow_right;
  int limiting;              /* Euler: modal-decay + characteristic WENO + positivity */
  double sensor_threshold;   /* default 1e-3 */
  double density_floor;      /* default 1e-10 */
  double pressure_floor;     /* default 1e-10 */
  int precision;             /* enum wasl_precision */
  int device;                /* CUDA device ordinal */
  int volume_rule_order;     /* mixed form: order r of the collapsed (r+1)^2-point volume
                                rule, p..p+2; 0 = p+2, the reference residual's rule;
                                -1 = the fully symmetric rule of degree 2p (3, 6, 12
                                points at P1, P2, P3) */
  int mixed_kernel;          /* mixed form: 0 autotuned; 1 face-centric kernels (face pass
                                + element pass); 2 + s the fused tile kernel in launch
                                shape s (0..13, see wasl_gpu_tuning) */
  int positivity_all;        /* with limiting: 1 applies the positivity limiter to every
                                element, not only troubled ones (not the reference's
                                behaviour, cpp/src/limiting/euler_modal_limiter.cpp:81-96) */
  int element_order;         /* 2D Euler mixed form: 0 stores the elements along a Morton
                                curve of their centroids (tiles of consecutive elements
                                are compact), 1 in the caller's order.  Either way every
                                face and element computes the same bits, and every call
                                that takes or returns per-element data uses the caller's
                                order; only wasl_gpu_state_device exposes the storage
                                order (wasl_gpu_element_order) */
} wasl_gpu_config;

/* Fill the reference's defaults (crates/wasl-bridge/src/config.rs:87-104). */
void wasl_gpu_config_default(wasl_gpu_config *config);

/* 1 when the library implements `precision` (enum wasl_precision) for this
 * dimension, equation and polynomial order, else 0. */
int wasl_gpu_form_supported(int precision, int dimensions, int equation, int polynomial_order);

/* Build the solver on a mesh given as node tags, coordinates ([node][dimensions])
 * and element connectivity ([element][dimensions+1] node tags).  The mesh is
 * normalized exactly as the reference normalizes it, so element order is the
 * caller's and face order is the reference's. */
int wasl_gpu_create(const wasl_gpu_config *config, int64_t node_count, const int64_t *node_tags,
                    const double *node_coordinates, int64_t element_count,
                    const int64_t *element_nodes, wasl_gpu **handle, char *error,
                    size_t error_length);

/* wasl_gpu_create on one part of a partitioned periodic triangle mesh (a
 * rank's owned elements and ghost layers): the periodic faces are given
 * instead of found by the donor search, since the part's own boundary also
 * holds the faces where its ghost region ends.  Per boundary face b of the
 * part's mesh (ascending face index, the faces without a second element) and
 * edge point q (p + 1 Gauss points): boundary_donors[b][q], the donor element
 * (an index into the part's elements), and boundary_basis[b][q][mode], the
 * donor's basis at the point's periodic image (wasl_mesh_periodic_trace of
 * the whole mesh gives both); donor -1 on every point of a face takes the
 * face's own element's trace (a cut face, whose neighbours are spoiled by
 * design).  config->boundary_left must be WASL_PERIODIC; 2D only.  The
 * reference distributes its meshes with MPI halos instead
 * (cpp/src/case/scalar_advection_distributed.cpp). */
int wasl_gpu_create_part(const wasl_gpu_config *config, int64_t node_count,
                         const int64_t *node_tags, const double *node_coordinates,
                         int64_t element_count, const int64_t *element_nodes,
                         int64_t boundary_faces, const int32_t *boundary_donors,
                         const double *boundary_basis, wasl_gpu **handle, char *error,
                         size_t error_length);

/* The periodic trace of a whole triangle mesh, without a handle (host
 * only): for every boundary face b (ascending face index) its element and
 * local edge (element[b], edge[b], in the normalized mesh: counter-clockwise
 * elements), and per edge point q the donor element donors[b][q] and the
 * donor's basis basis[b][q][mode] at the point's periodic image.  Call with
 * element == NULL to get the boundary face count in *boundary_faces, then
 * with arrays sized from it.  The reference's
 * cpp/src/boundaries/periodic_triangle_trace.cpp:40-67. */
int wasl_mesh_periodic_trace(int64_t node_count, const int64_t *node_tags,
                             const double *node_coordinates, int64_t element_count,
                             const int64_t *element_nodes, int polynomial_order,
                             int64_t *boundary_faces, int32_t *element, int32_t *edge,
                             int32_t *donors, double *basis, char *error, size_t error_length);
void wasl_gpu_destroy(wasl_gpu *handle);
const char *wasl_gpu_last_error(const wasl_gpu *handle);

/* Counts: elements, faces, modes per variable, variables. */
int wasl_gpu_sizes(const wasl_gpu *handle, int64_t *elements, int64_t *faces, int *modes,
                   int *variables);

/* Element geometry after normalization: [element][6] vertices (2D) or
 * [element][2] ends (1D). */
int wasl_gpu_element_vertices(const wasl_gpu *handle, double *vertices, int64_t count);

/* Modal state in the checkpoint layout U[variable][mode][element], FP64. */
int wasl_gpu_set_state(wasl_gpu *handle, const double *coefficients, int64_t count);
int wasl_gpu_get_state(wasl_gpu *handle, double *coefficients, int64_t count);

/* Quadrature of rule order r (the collapsed (r+1)^2-point triangle rule, or
 * the (r+1)-point Gauss rule on lines): physical points and physical weights
 * (reference weight x |det J|), packed [element][point]; y may be NULL in 1D.
 * wasl_gpu_rule_points gives the points per element. */
int wasl_gpu_rule_points(const wasl_gpu *handle, int rule_order, int *points);
int wasl_gpu_quadrature(const wasl_gpu *handle, int rule_order, double *x, double *y,
                        double *weights);

/* Initial state by L2 projection of point values [element][point][variable]
 * at the rule's points (cpp/include/wasl/dg/l2_projection.hpp:36-76;
 * cpp/src/case/initial_state.cpp:16-64 uses rule order max(p, 5) on triangles
 * and 7 Gauss points on lines). */
int wasl_gpu_project(wasl_gpu *handle, int rule_order, const double *values, int64_t count);

/* The state evaluated at the rule's points, [element][point][variable]. */
int wasl_gpu_evaluate(wasl_gpu *handle, int rule_order, double *values, int64_t count);

/* CFL time step of the current state, bit-identical to the reference's
 * (the device finds the fastest cell, the host evaluates its speed). */
int wasl_gpu_stable_dt(wasl_gpu *handle, double cfl, double *dt);

/* The two factors of that time step, dt = cfl * length / (speed * (2p + 1)):
 * the largest cell-average wave speed (hypot(u, v) + c, evaluated as
 * wasl_gpu_stable_dt evaluates it) and the smallest element length (the
 * smallest altitude, cpp/src/time/cfl_timestep.cpp:22-30, 70-84).  A run
 * partitioned over ranks reduces speed by max and length by min and forms the
 * dt of one solver over the whole mesh (2D Euler only). */
int wasl_gpu_cfl_parts(wasl_gpu *handle, double *speed, double *length);

/* One SSP-RK3 step with the stage limiter (when enabled). */
int wasl_gpu_step(wasl_gpu *handle, double dt);

/* The stage limiter applied to the current state, as the reference applies it
 * to the projected initial state (cpp/src/case/euler_triangle.cpp:33-37).
 * No-op without limiting. */
int wasl_gpu_limit(wasl_gpu *handle);

/* Troubled-cell flags of the three stages of the last step, [stage][element]. */
int wasl_gpu_get_flags(wasl_gpu *handle, uint8_t *flags, int64_t count);

/* Totals of density and energy: sum over elements of sqrt(2) det(J) c0
 * (cpp/src/case/euler_diagnostics.cpp:26-39); scalar: energy = mass. */
int wasl_gpu_mass_energy(wasl_gpu *handle, double *mass, double *energy);

/* The serial run loop: dt = stable_dt clipped to land on end_time, advance,
 * until end_time or max_steps (serial_case_runner.cpp:107-149). */
int wasl_gpu_run(wasl_gpu *handle, double cfl, double start_time, double end_time,
                 uint64_t max_steps, uint64_t *steps, double *time);

/* wasl_gpu_run in one kernel launch with no host round trip per step: the
 * same loop, dt and results bit for bit, for line meshes whose state (three
 * buffers of variables x modes x elements doubles, at most 200 KiB) fits in
 * one CTA's shared memory, without the limiter (the 400-cell P2 advection
 * run, for one).  WASL_ERR_ARGUMENT otherwise.  No counterpart in the
 * reference (its loop is the host loop wasl_gpu_run mirrors). */
int wasl_gpu_run_resident(wasl_gpu *handle, double cfl, double start_time, double end_time,
                          uint64_t max_steps, uint64_t *steps, double *time);

/* Device-resident fast path: `steps` steps with the CFL step computed on the
 * device each step, enqueued on the handle's stream without host
 * synchronization; a device error (non-physical average, positivity floor)
 * is raised by wasl_gpu_sync or the next call that waits for the device. */
int wasl_gpu_advance(wasl_gpu *handle, double cfl, int64_t steps);

/* Waits for the handle's stream and reports a pending device error. */
int wasl_gpu_sync(wasl_gpu *handle);

/* The mixed form's kernel in use: 0 face-centric kernels, 1 + s the fused
 * tile kernel in launch shape s (0: 128 elements per CTA at <= 128 registers
 * a thread; 1: 128, no register cap; 2: 256 at <= 128; 3: 64 at <= 128;
 * 4-7: the shared-face tile kernel, which evaluates a face between two
 * elements of one tile once: 4: 64 elements per CTA sized for 7 CTAs per SM;
 * 5: 96 for 5; 6: 128 for 4; 7: 128 for 3; 8-11: the patch kernel, which
 * evaluates each element's traces once and each face inside a patch once,
 * without the limiter only: 8: 128 elements per CTA at <= 128 registers;
 * 9: 128 sized for 5 CTAs per SM; 10: 64 for 8; 11: 64 for 10; 12-13: the
 * patch kernel with its volume contractions on the tensor cores (split-TF32
 * mma.sync, FP32 accumulation): 12: 128 at <= 128 registers, 13: 128 for 5);
 * -1 for forms with a single kernel or before the first step.  When the
 * choice was autotuned (mixed_kernel 0: every variant timed on the solver's
 * own state before its first step, the fastest kept for the process per
 * polynomial order, rule order and mesh size class), `ms` receives up to
 * `capacity` per-variant stage times and `count` their number. */
int wasl_gpu_tuning(const wasl_gpu *handle, int *choice, double *ms, int capacity, int *count);

/* The storage order of the device state (wasl_gpu_state_device): order[i] is
 * the caller's element stored at column i (count = element count).  The
 * identity except for the 2D Euler mixed form with element_order 0.  No
 * counterpart in the reference (its state lives in host vectors). */
int wasl_gpu_element_order(const wasl_gpu *handle, int64_t *order, int64_t count);

/* Setup phases timed by wasl_gpu_create (wall clock, ms), for
 * wasl_gpu_setup_times.  The reference builds the same data in its case
 * drivers (cpp/src/case/euler_triangle.cpp:16-25). */
enum wasl_setup_phase {
  WASL_SETUP_TOPOLOGY = 0, /* mesh normalisation and faces (host) */
  WASL_SETUP_ORDER = 1,    /* element storage order (host) */
  WASL_SETUP_PERIODIC = 2, /* periodic donor search (device) and donor basis (host) */
  WASL_SETUP_FACES = 3,    /* face slots, tile and patch arrays, reference tables */
  WASL_SETUP_STENCIL = 4,  /* limiter stencil: neighbours (host), transforms (device) */
  WASL_SETUP_OTHER = 5,    /* state buffers and the remaining uploads */
  WASL_SETUP_PHASES = 6
};
/* The setup phases' times: ms[phase] for phase < count (count <= 6).  Phases
 * a solver has no work for read 0. */
int wasl_gpu_setup_times(const wasl_gpu *handle, double *ms, int count);

/* The limiter stencil's candidate transforms as the limiter reads them,
 * [element][candidate][target mode][source mode] in the caller's order
 * (count = elements x 3 x modes^2), built on the device at setup.  Matches
 * the reference's CandidateTransform (cpp/include/wasl/limiting/weno/
 * candidate_transform.hpp:18-41).  2D Euler with limiting only. */
int wasl_gpu_stencil_transforms(wasl_gpu *handle, double *transforms, int64_t count);

/* The periodic trace as the stage kernels read it: for every boundary face
 * b (ascending face index) and edge point q, the donor element (caller's
 * index) and the donor's basis at the image point, donors [b][q], basis
 * [b][q][mode] (points = boundary faces x (p + 1)).  Matches the reference's
 * periodic trace (cpp/src/boundaries/periodic_triangle_trace.cpp:40-67).
 * Periodic triangle meshes only. */
int wasl_gpu_periodic_trace(wasl_gpu *handle, int32_t *donors, double *basis, int64_t points);

/* ---- halo exchange of a partitioned run (one rank per GPU) ----------------
 *
 * A rank holds its part of the mesh (owned elements and ghost layers) on one
 * handle; per peer rank, the halo schedule lists the owned elements the peer
 * imports (sends) and the ghosts imported from it (receives), each ascending
 * (cpp/include/wasl/communication/halo_schedule.hpp:17-42).  The halo packs
 * a peer's send columns into one [rows][count] device buffer, unpacks a
 * receive buffer into the ghost columns (rows = variables x modes), and moves
 * the buffers over NCCL, or leaves them to the caller's transport
 * (wasl_halo_buffers).  All work runs on the handle's stream.  Element
 * indices are the handle's (caller's) element indices. */
typedef struct wasl_halo wasl_halo;

/* peers: count of peer ranks; peer_ranks[k]: the k-th peer's rank;
 * send_counts[k] / recv_counts[k]: its list lengths; send_elements /
 * recv_elements: the lists, peer after peer. */
int wasl_halo_create(wasl_gpu *handle, int peers, const int32_t *peer_ranks,
                     const int64_t *send_counts, const int64_t *send_elements,
                     const int64_t *recv_counts, const int64_t *recv_elements, wasl_halo **halo,
                     char *error, size_t error_length);
void wasl_halo_destroy(wasl_halo *halo);
const char *wasl_halo_last_error(const wasl_halo *halo);
int wasl_halo_pack(wasl_halo *halo);
int wasl_halo_unpack(wasl_halo *halo);
/* Peer k's device buffers ([rows][count] doubles), counts and rows. */
int wasl_halo_buffers(wasl_halo *halo, int peer, double **send, double **recv,
                      int64_t *send_count, int64_t *recv_count, int64_t *rows);
/* pack, one NCCL group of a send and a receive per peer (comm: an
 * ncclComm_t of the run's ranks), unpack; returns when enqueued. */
int wasl_halo_exchange_nccl(wasl_halo *halo, void *comm);
/* The whole mesh's CFL step: the handle's CFL parts all-reduced (largest
 * speed, smallest length) over comm, then stable_dt's formula (2D Euler). */
int wasl_gpu_stable_dt_nccl(wasl_gpu *handle, void *comm, double cfl, double *dt);
/* NCCL communicators for callers without their own: an id made on one rank
 * and shared with the others, then one communicator per rank. */
int wasl_nccl_unique_id(uint8_t *id /* 128 bytes */);
int wasl_nccl_comm_create(int ranks, const uint8_t *id, int rank, int device, void **comm,
                          char *error, size_t error_length);
void wasl_nccl_comm_destroy(void *comm);

/* Device pointer of the state U[variable][mode][element] and the handle's
 * CUDA stream (cudaStream_t), for callers that keep data on the device. */
int wasl_gpu_state_device(wasl_gpu *handle, double **device_pointer);
int wasl_gpu_stream(wasl_gpu *handle, void **stream);

/* Measurement hooks: profile_begin zeroes the launch counter and brackets
 * every following stage kernel with CUDA events on the handle's stream;
 * profile_end synchronizes and returns the summed stage-kernel time (ms), the
 * number of stage kernels timed, and all kernels launched since begin. */
int wasl_gpu_profile_begin(wasl_gpu *handle);
int wasl_gpu_profile_end(wasl_gpu *handle, double *stage_kernel_ms, int64_t *stage_kernels,
                         int64_t *kernel_launches);
/* The stage-kernel time of the last profile_end split by SSP-RK3 stage:
 * stage_ms[k] sums the timed kernels of stage k (0, 1, 2) of every step. */
int wasl_gpu_profile_stages(const wasl_gpu *handle, double *stage_ms);

/* Restart files with the fields of the reference Checkpoint
 * (cpp/include/wasl/io/checkpoint.hpp:17-29) in a portable binary container
 * (HDF5 is not available here). */
int wasl_gpu_write_checkpoint(wasl_gpu *handle, const char *path, double time, uint64_t step,
                              const char *prepared_mesh);
int wasl_gpu_read_checkpoint(wasl_gpu *handle, const char *path, double *time, uint64_t *step);

/* ---- Learned troubled-cell indicator -----------------------------------------
 * A small network (features -> 64 -> 64 -> 1, BF16 weights, FP32 accumulate)
 * over the normalised density modes of a cell and its three limiter-stencil
 * neighbours, trained on the flags of the reference modal-decay sensor
 * (cpp/src/limiting/euler_modal_limiter.cpp:18-24) on the method's own runs.
 * With it set, each stage's troubled cells are the network's decision where
 * sigmoid(logit) >= hi or <= lo, and the reference sensor's elsewhere (the
 * fallback); the limiter then runs as usual.  No counterpart in the reference.
 * 2D Euler with limiting only. */

/* Features per element for this solver: 4 (M - 1) + 3, padded to 16k. */
int wasl_gpu_indicator_features(const wasl_gpu *handle, int *features);

/* The current state's features [element][features] and the reference
 * sensor's flags [element] (training data). */
int wasl_gpu_indicator_data(wasl_gpu *handle, float *features, uint8_t *labels, int64_t count);

/* The learned indicator's inference kernel: 0 (the default) the tcgen05
 * tensor cores (single-CTA MMAs of 128 rows, accumulators in TMEM), 1 the
 * warp-level mma.sync kernel; both give the same decisions up to the FP32
 * rounding of the accumulation order.  No counterpart in the reference. */
int wasl_gpu_indicator_kernel(wasl_gpu *handle, int kernel);

/* Use the network with FP32 weights (wasl_mlp_get_weights layout) and the
 * confidence band (lo, hi) handed to the reference sensor (lo < 0 and hi > 1:
 * every cell falls back, which reproduces the reference sensor exactly). */
int wasl_gpu_set_indicator(wasl_gpu *handle, const float *weights, int64_t count, double lo,
                           double hi);

/* The network's logits for the current state (the tensor-core inference
 * kernel), one per element. */
int wasl_gpu_indicator_logits(wasl_gpu *handle, float *logits, int64_t count);

/* Cell-stage counts since the indicator was set (or last reset): [0] network
 * troubled, [1] network smooth, [2] fallback to the reference, [3] reference
 * troubled, [4] missed (reference troubled, decided smooth), [5] false
 * (reference smooth, decided troubled). */
int wasl_gpu_indicator_stats(wasl_gpu *handle, uint64_t *stats, int reset);

/* Training on the GPU (the project's own forward/backward and Adam kernels). */
typedef struct wasl_mlp wasl_mlp;
int wasl_mlp_create(int features, uint64_t seed, int device, wasl_mlp **handle, char *error,
                    size_t error_length);
void wasl_mlp_destroy(wasl_mlp *handle);
const char *wasl_mlp_last_error(const wasl_mlp *handle);
int wasl_mlp_parameter_count(const wasl_mlp *handle, int64_t *count);
/* Training samples [sample][features] and 0/1 labels, copied to the device. */
int wasl_mlp_set_data(wasl_mlp *handle, const float *features, const uint8_t *labels,
                      int64_t count);
/* `steps` Adam steps (lr, beta 0.9/0.999) on mini-batches of `batch` samples
 * (a multiple of 64) taken in order, cycling; loss: weighted binary
 * cross-entropy (positives weighted positive_weight), mean of the last batch. */
int wasl_mlp_train(wasl_mlp *handle, int64_t steps, int64_t batch, double learning_rate,
                   double positive_weight, double *loss);
/* The gradient of the mean loss over `count` samples (a multiple of 64) at the
 * current weights, in the weights' layout, and that loss. */
int wasl_mlp_gradient(wasl_mlp *handle, const float *features, const uint8_t *labels,
                      int64_t count, double positive_weight, float *gradient, double *loss);
int wasl_mlp_predict(wasl_mlp *handle, const float *features, int64_t count, float *logits);
/* FP32 weights: W1 [64][F], b1 [64], W2 [64][64], b2 [64], w3 [64], b3. */
int wasl_mlp_get_weights(const wasl_mlp *handle, float *weights, int64_t count);
int wasl_mlp_set_weights(wasl_mlp *handle, const float *weights, int64_t count);

/* ---- Batched 2D Euler (the mixed form) --------------------------------------
 * Many independent triangle meshes of uneven size and polynomial order (1-3)
 * advanced together: cases of one order share one launch of the fused tile
 * kernel per stage over a work list of element tiles (tiles never straddle
 * cases, each carries its case's own CFL time step), and a step (per-case CFL,
 * three stages, stage limiter) is captured once in a CUDA graph and replayed.
 * No counterpart in the reference, which runs one case per process
 * (cpp/src/case/serial_case_runner.cpp:117-149); each case behaves as that
 * loop's case with the mixed form's arithmetic. */
typedef struct wasl_batch wasl_batch;

typedef struct {
  double heat_capacity_ratio;
  int boundary;              /* WASL_PERIODIC (faces must pair) or WASL_TRANSMISSIVE */
  int limiting;              /* modal-decay sensor + characteristic WENO + positivity */
  double sensor_threshold;
  double density_floor;
  double pressure_floor;
  int reduced_volume_rule;   /* 1: volume rule order p; 0: p+2 (the reference's rule) */
  int tile_shape;            /* 0 autotuned per polynomial order; 1 + s launch shape s */
  int use_graph;             /* 1: capture the step in a CUDA graph and replay it */
  int device;
  int positivity_all;        /* with limiting: positivity limiter on every element */
} wasl_batch_config;

void wasl_batch_config_default(wasl_batch_config *config);

/* Cases are given back to back: orders[c], node_counts[c] node tags and
 * [node][2] coordinates, element_counts[c] triangles ([element][3] node tags). */
int wasl_batch_create(const wasl_batch_config *config, int64_t case_count, const int *orders,
                      const int64_t *node_counts, const int64_t *node_tags,
                      const double *node_coordinates, const int64_t *element_counts,
                      const int64_t *element_nodes, wasl_batch **handle, char *error,
                      size_t error_length);
void wasl_batch_destroy(wasl_batch *handle);
const char *wasl_batch_last_error(const wasl_batch *handle);

/* Totals over all cases, and one case's elements and modes per variable. */
int wasl_batch_sizes(const wasl_batch *handle, int64_t *cases, int64_t *elements, int64_t *dof);
int wasl_batch_case_size(const wasl_batch *handle, int64_t case_index, int64_t *elements,
                         int *modes);

/* One case's state U[variable][mode][element] (FP64, that case's elements). */
int wasl_batch_set_state(wasl_batch *handle, int64_t case_index, const double *coefficients,
                         int64_t count);
int wasl_batch_get_state(wasl_batch *handle, int64_t case_index, double *coefficients,
                         int64_t count);

/* Quadrature and L2 projection of one case, as wasl_gpu_quadrature and
 * wasl_gpu_project. */
int wasl_batch_quadrature(const wasl_batch *handle, int64_t case_index, int rule_order, double *x,
                          double *y, double *weights);
int wasl_batch_project(wasl_batch *handle, int64_t case_index, int rule_order,
                       const double *values, int64_t count);

/* The stage limiter applied to every case's current state, as the reference
 * applies it to the projected initial state (cpp/src/case/euler_triangle.cpp:33-37).
 * No-op without limiting. */
int wasl_batch_limit(wasl_batch *handle);

/* `steps` SSP-RK3 steps of every case, each with its own CFL time step
 * cfl h_c / ((|u| + c)_max,c (2 p_c + 1)).  A case that fails (a non-physical
 * cell average, or a mean below a positivity floor) is frozen (dt 0 from then
 * on) and recorded in wasl_batch_status; the other cases go on, and the call
 * still returns 0.  Synchronizes to report CUDA errors. */
int wasl_batch_advance(wasl_batch *handle, double cfl, int64_t steps);

/* Per case: 0, or the failure that froze it: 1 a non-physical cell average
 * (cpp/src/time/cfl_timestep.cpp:39-40), 2 a positivity mean below a floor
 * (cpp/include/wasl/limiting/positivity/euler_positivity.hpp:74-75). */
int wasl_batch_status(wasl_batch *handle, int *status, int64_t count);

/* Per case: time advanced since creation, and the last step's dt. */
int wasl_batch_times(wasl_batch *handle, double *time, double *dt, int64_t count);

/* The tile shape chosen for the cases of order p (-1 if none), and the timed
 * mean stage time of every shape when it was autotuned. */
int wasl_batch_tuning(const wasl_batch *handle, int polynomial_order, int *choice, double *ms,
                      int capacity, int *count);

/* Kernels enqueued per step, whether steps replay a CUDA graph, all kernels
 * launched so far, and the handle's CUDA stream (cudaStream_t). */
int wasl_batch_launches(const wasl_batch *handle, int64_t *per_step, int *graph, int64_t *total);
int wasl_batch_stream(wasl_batch *handle, void **stream);

/* The CFL time step of a device-resident 2D/1D Euler state, computed without
 * allocating anything.  No counterpart in the reference: it is an entry point
 * for callers that cannot call cudaMalloc (an application whose device memory
 * is owned by its own pool allocator, or a latency-critical loop that cannot
 * take cudaMalloc's implicit device synchronization).  `state` is
 * U[variable][mode][element] in device memory, `length` the mesh's smallest
 * altitude (or length in 1D), `dt` one double of device memory that receives
 * cfl * length / (max |u|+c over cell averages * (2p+1)), or 0 when that speed
 * is 0: the value wasl_gpu_stable_dt gives for the same state, bit for bit;
 * `stream` a cudaStream_t (NULL: the default stream).  The reduction's
 * scratch is a fixed 9.6 KiB array that every GPU loading the library holds
 * until exit; element_count above 2,147,483,647 is rejected.  Every call
 * shares that array, so calls whose kernels overlap on one GPU race.  The
 * first call on a device looks up the array's address with that device
 * current.  Every call copies the result through the host and synchronizes
 * `stream`, so it cannot be called while that stream is being captured.  It
 * returns WASL_ERR_NONPHYSICAL for a non-physical cell average, with the
 * message in `error`. */
int wasl_cfl_dt_static(const double *state, int64_t element_count, int mode_count, int dimensions,
                       int polynomial_order, double gamma, double cfl, double length, double *dt,
                       void *stream, char *error, size_t error_length);

#ifdef __cplusplus
}
#endif

#endif
