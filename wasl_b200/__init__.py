"""B200-native modal RKDG time step for the Wasl solver (scalar advection and
compressible Euler on 1D line and 2D triangle meshes).

The numerical work runs in ``libwasl_b200.so`` (CUDA kernels for sm_100a behind
the C-ABI declared in ``include/wasl_b200.h``).  This module is a thin ctypes
mirror of the reference's case-model interface
(cpp/include/wasl/case/serial_case_runner.hpp:22-34):

    Solver.set_state / get_state     initial_state, from_checkpoint / to_checkpoint
    Solver.stable_dt                 stable_time_step
    Solver.step                      advance (one SSP-RK3 step with the stage limiter)
    Solver.mass_energy               mass
    Solver.run                       the run_serial_case loop
    Solver.write_checkpoint / read_checkpoint

There is no CPU fallback: constructing a Solver without the built library or
without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# WASL_B200_LIBRARY selects another build of the library (the checked build,
# libwasl_b200_checked.so, for one).
LIB_PATH = os.environ.get("WASL_B200_LIBRARY", os.path.join(HERE, "libwasl_b200.so"))

PERIODIC, INFLOW, OUTFLOW, TRANSMISSIVE = 0, 1, 2, 3
SCALAR_ADVECTION, EULER = 0, 1
PLAIN_FP64, MIXED = 0, 1
BOUNDARY_KINDS = {"periodic": PERIODIC, "inflow": INFLOW, "outflow": OUTFLOW,
                  "transmissive": TRANSMISSIVE}
PRECISIONS = {"plain": PLAIN_FP64, "fp64": PLAIN_FP64, "mixed": MIXED}


class WaslError(RuntimeError):
    """A failure reported by the library; ``status`` is the C-ABI status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class Config(C.Structure):
    _fields_ = [
        ("dimensions", C.c_int), ("equation", C.c_int), ("polynomial_order", C.c_int),
        ("heat_capacity_ratio", C.c_double), ("velocity_x", C.c_double),
        ("velocity_y", C.c_double), ("boundary_left", C.c_int), ("boundary_right", C.c_int),
        ("inflow_left", C.c_double), ("inflow_right", C.c_double), ("limiting", C.c_int),
        ("sensor_threshold", C.c_double), ("density_floor", C.c_double),
        ("pressure_floor", C.c_double), ("precision", C.c_int), ("device", C.c_int),
        ("volume_rule_order", C.c_int), ("mixed_kernel", C.c_int),
        ("positivity_all", C.c_int), ("element_order", C.c_int),
    ]


class BatchConfig(C.Structure):
    _fields_ = [
        ("heat_capacity_ratio", C.c_double), ("boundary", C.c_int), ("limiting", C.c_int),
        ("sensor_threshold", C.c_double), ("density_floor", C.c_double),
        ("pressure_floor", C.c_double), ("reduced_volume_rule", C.c_int),
        ("tile_shape", C.c_int), ("use_graph", C.c_int), ("device", C.c_int),
        ("positivity_all", C.c_int),
    ]


_d = C.POINTER(C.c_double)
_i64 = C.POINTER(C.c_int64)
_u8 = C.POINTER(C.c_uint8)
_f = C.POINTER(C.c_float)
_lib = None

# name -> (restype, argtypes), one per declaration in include/wasl_b200.h
SIGNATURES = {
    "wasl_gpu_config_default": (None, [C.POINTER(Config)]),
    "wasl_gpu_create": (C.c_int, [C.POINTER(Config), C.c_int64, _i64, _d, C.c_int64, _i64,
                                  C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "wasl_gpu_create_part": (C.c_int, [C.POINTER(Config), C.c_int64, _i64, _d, C.c_int64, _i64,
                                       C.c_int64, C.POINTER(C.c_int32), _d,
                                       C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "wasl_mesh_periodic_trace": (C.c_int, [C.c_int64, _i64, _d, C.c_int64, _i64, C.c_int, _i64,
                                           C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                           C.POINTER(C.c_int32), _d, C.c_char_p, C.c_size_t]),
    "wasl_gpu_form_supported": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int]),
    "wasl_halo_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int32), _i64, _i64, _i64,
                                   _i64, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "wasl_halo_destroy": (None, [C.c_void_p]),
    "wasl_halo_last_error": (C.c_char_p, [C.c_void_p]),
    "wasl_halo_pack": (C.c_int, [C.c_void_p]),
    "wasl_halo_unpack": (C.c_int, [C.c_void_p]),
    "wasl_halo_buffers": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_void_p), _i64, _i64, _i64]),
    "wasl_halo_exchange_nccl": (C.c_int, [C.c_void_p, C.c_void_p]),
    "wasl_gpu_stable_dt_nccl": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, _d]),
    "wasl_nccl_unique_id": (C.c_int, [C.POINTER(C.c_uint8)]),
    "wasl_nccl_comm_create": (C.c_int, [C.c_int, C.POINTER(C.c_uint8), C.c_int, C.c_int,
                                        C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "wasl_nccl_comm_destroy": (None, [C.c_void_p]),
    "wasl_gpu_destroy": (None, [C.c_void_p]),
    "wasl_gpu_last_error": (C.c_char_p, [C.c_void_p]),
    "wasl_gpu_sizes": (C.c_int, [C.c_void_p, _i64, _i64, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)]),
    "wasl_gpu_element_vertices": (C.c_int, [C.c_void_p, _d, C.c_int64]),
    "wasl_gpu_set_state": (C.c_int, [C.c_void_p, _d, C.c_int64]),
    "wasl_gpu_get_state": (C.c_int, [C.c_void_p, _d, C.c_int64]),
    "wasl_gpu_rule_points": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "wasl_gpu_quadrature": (C.c_int, [C.c_void_p, C.c_int, _d, _d, _d]),
    "wasl_gpu_project": (C.c_int, [C.c_void_p, C.c_int, _d, C.c_int64]),
    "wasl_gpu_evaluate": (C.c_int, [C.c_void_p, C.c_int, _d, C.c_int64]),
    "wasl_gpu_stable_dt": (C.c_int, [C.c_void_p, C.c_double, _d]),
    "wasl_gpu_step": (C.c_int, [C.c_void_p, C.c_double]),
    "wasl_gpu_limit": (C.c_int, [C.c_void_p]),
    "wasl_gpu_get_flags": (C.c_int, [C.c_void_p, _u8, C.c_int64]),
    "wasl_gpu_mass_energy": (C.c_int, [C.c_void_p, _d, _d]),
    "wasl_gpu_run": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_uint64,
                               C.POINTER(C.c_uint64), _d]),
    "wasl_gpu_run_resident": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                        C.c_uint64, C.POINTER(C.c_uint64), _d]),
    "wasl_gpu_advance": (C.c_int, [C.c_void_p, C.c_double, C.c_int64]),
    "wasl_gpu_sync": (C.c_int, [C.c_void_p]),
    "wasl_gpu_state_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "wasl_gpu_element_order": (C.c_int, [C.c_void_p, _i64, C.c_int64]),
    "wasl_gpu_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "wasl_gpu_setup_times": (C.c_int, [C.c_void_p, _d, C.c_int]),
    "wasl_gpu_stencil_transforms": (C.c_int, [C.c_void_p, _d, C.c_int64]),
    "wasl_gpu_periodic_trace": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), _d, C.c_int64]),
    "wasl_gpu_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), _d, C.c_int,
                                  C.POINTER(C.c_int)]),
    "wasl_batch_config_default": (None, [C.POINTER(BatchConfig)]),
    "wasl_batch_create": (C.c_int, [C.POINTER(BatchConfig), C.c_int64, C.POINTER(C.c_int), _i64,
                                    _i64, _d, _i64, _i64, C.POINTER(C.c_void_p), C.c_char_p,
                                    C.c_size_t]),
    "wasl_batch_destroy": (None, [C.c_void_p]),
    "wasl_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "wasl_batch_sizes": (C.c_int, [C.c_void_p, _i64, _i64, _i64]),
    "wasl_batch_case_size": (C.c_int, [C.c_void_p, C.c_int64, _i64, C.POINTER(C.c_int)]),
    "wasl_batch_set_state": (C.c_int, [C.c_void_p, C.c_int64, _d, C.c_int64]),
    "wasl_batch_get_state": (C.c_int, [C.c_void_p, C.c_int64, _d, C.c_int64]),
    "wasl_batch_quadrature": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, _d, _d, _d]),
    "wasl_batch_project": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, _d, C.c_int64]),
    "wasl_batch_limit": (C.c_int, [C.c_void_p]),
    "wasl_batch_advance": (C.c_int, [C.c_void_p, C.c_double, C.c_int64]),
    "wasl_batch_times": (C.c_int, [C.c_void_p, _d, _d, C.c_int64]),
    "wasl_batch_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_int64]),
    "wasl_batch_tuning": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), _d, C.c_int,
                                    C.POINTER(C.c_int)]),
    "wasl_batch_launches": (C.c_int, [C.c_void_p, _i64, C.POINTER(C.c_int), _i64]),
    "wasl_batch_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "wasl_gpu_indicator_features": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "wasl_gpu_indicator_data": (C.c_int, [C.c_void_p, _f, _u8, C.c_int64]),
    "wasl_gpu_set_indicator": (C.c_int, [C.c_void_p, _f, C.c_int64, C.c_double, C.c_double]),
    "wasl_gpu_indicator_kernel": (C.c_int, [C.c_void_p, C.c_int]),
    "wasl_gpu_indicator_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.c_int]),
    "wasl_gpu_indicator_logits": (C.c_int, [C.c_void_p, _f, C.c_int64]),
    "wasl_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_void_p),
                                  C.c_char_p, C.c_size_t]),
    "wasl_mlp_destroy": (None, [C.c_void_p]),
    "wasl_mlp_last_error": (C.c_char_p, [C.c_void_p]),
    "wasl_mlp_parameter_count": (C.c_int, [C.c_void_p, _i64]),
    "wasl_mlp_set_data": (C.c_int, [C.c_void_p, _f, _u8, C.c_int64]),
    "wasl_mlp_train": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_double, C.c_double, _d]),
    "wasl_mlp_gradient": (C.c_int, [C.c_void_p, _f, _u8, C.c_int64, C.c_double, _f, _d]),
    "wasl_mlp_predict": (C.c_int, [C.c_void_p, _f, C.c_int64, _f]),
    "wasl_mlp_get_weights": (C.c_int, [C.c_void_p, _f, C.c_int64]),
    "wasl_mlp_set_weights": (C.c_int, [C.c_void_p, _f, C.c_int64]),
    "wasl_gpu_profile_begin": (C.c_int, [C.c_void_p]),
    "wasl_gpu_profile_end": (C.c_int, [C.c_void_p, _d, _i64, _i64]),
    "wasl_gpu_profile_stages": (C.c_int, [C.c_void_p, _d]),
    "wasl_gpu_cfl_parts": (C.c_int, [C.c_void_p, _d, _d]),
    "wasl_gpu_write_checkpoint": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_uint64,
                                            C.c_char_p]),
    "wasl_gpu_read_checkpoint": (C.c_int, [C.c_void_p, C.c_char_p, _d,
                                           C.POINTER(C.c_uint64)]),
    "wasl_cfl_dt_static": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int,
                                     C.c_double, C.c_double, C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_char_p, C.c_size_t]),
}


def library(path: str = LIB_PATH):
    """Load libwasl_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m wasl_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def form_available(precision: str, dimensions: int = 2, equation: str = "euler",
                   polynomial_order: int = 2) -> bool:
    """Whether the library implements a precision form for this case."""
    return bool(library().wasl_gpu_form_supported(
        PRECISIONS[precision], dimensions, EULER if equation == "euler" else SCALAR_ADVECTION,
        polynomial_order))


def _ptr(a, t=_d):
    return a.ctypes.data_as(t)


def default_config() -> Config:
    cfg = Config()
    library().wasl_gpu_config_default(C.byref(cfg))
    return cfg


def mesh_periodic_trace(node_tags, node_coordinates, element_nodes, polynomial_order):
    """The periodic trace of a whole triangle mesh (wasl_mesh_periodic_trace):
    (element [b], edge [b], donors [b][p+1], basis [b][p+1][modes]) for every
    boundary face b in ascending face order; edges are local edge indices of
    the counter-clockwise normalized element."""
    lib = library()
    tags = np.ascontiguousarray(node_tags, dtype=np.int64)
    coords = np.ascontiguousarray(node_coordinates, dtype=np.float64)
    elems = np.ascontiguousarray(element_nodes, dtype=np.int64)
    err = C.create_string_buffer(1024)
    count = C.c_int64()
    i32 = C.POINTER(C.c_int32)
    args = (len(tags), _ptr(tags, _i64), _ptr(coords), len(elems), _ptr(elems, _i64),
            polynomial_order)
    rc = lib.wasl_mesh_periodic_trace(*args, C.byref(count), None, None, None, None, err,
                                      len(err))
    if rc != 0:
        raise WaslError(rc, err.value.decode())
    b, Q = count.value, polynomial_order + 1
    M = (polynomial_order + 1) * (polynomial_order + 2) // 2
    element = np.empty(b, dtype=np.int32)
    edge = np.empty(b, dtype=np.int32)
    donors = np.empty((b, Q), dtype=np.int32)
    basis = np.empty((b, Q, M))
    rc = lib.wasl_mesh_periodic_trace(*args, C.byref(count), element.ctypes.data_as(i32),
                                      edge.ctypes.data_as(i32), donors.ctypes.data_as(i32),
                                      _ptr(basis), err, len(err))
    if rc != 0:
        raise WaslError(rc, err.value.decode())
    return element, edge, donors, basis


class Solver:
    """One mesh, one equation, one polynomial order, state resident on the GPU."""

    def __init__(self, node_tags, node_coordinates, element_nodes, *, dimensions=2,
                 equation="euler", polynomial_order=2, gamma=1.4, velocity=(0.0, 0.0),
                 boundary="periodic", boundary_right=None, inflow=(0.0, 0.0), limiting=False,
                 sensor_threshold=1e-3, density_floor=1e-10, pressure_floor=1e-10,
                 precision="plain", device=0, volume_rule_order=0, mixed_kernel=0,
                 positivity_all=False, element_order="curve", part_boundary=None):
        """part_boundary: (donors [b][p+1] int32, basis [b][p+1][modes]) for a
        part of a partitioned periodic mesh (wasl_gpu_create_part;
        halo.LocalMesh.part_boundary), None for a whole mesh."""
        lib = library()
        cfg = default_config()
        cfg.dimensions = dimensions
        cfg.equation = EULER if equation == "euler" else SCALAR_ADVECTION
        cfg.polynomial_order = polynomial_order
        cfg.heat_capacity_ratio = gamma
        cfg.velocity_x, cfg.velocity_y = velocity
        cfg.boundary_left = BOUNDARY_KINDS[boundary]
        cfg.boundary_right = BOUNDARY_KINDS[boundary_right or boundary]
        cfg.inflow_left, cfg.inflow_right = inflow
        cfg.limiting = 1 if limiting else 0
        cfg.sensor_threshold = sensor_threshold
        cfg.density_floor = density_floor
        cfg.pressure_floor = pressure_floor
        cfg.precision = PRECISIONS[precision]
        cfg.device = device
        cfg.volume_rule_order = volume_rule_order
        cfg.mixed_kernel = mixed_kernel
        cfg.positivity_all = 1 if positivity_all else 0
        cfg.element_order = {"curve": 0, "caller": 1}[element_order]
        self.config = cfg
        tags = np.ascontiguousarray(node_tags, dtype=np.int64)
        coords = np.ascontiguousarray(node_coordinates, dtype=np.float64)
        elems = np.ascontiguousarray(element_nodes, dtype=np.int64)
        err = C.create_string_buffer(1024)
        h = C.c_void_p()
        if part_boundary is None:
            rc = lib.wasl_gpu_create(C.byref(cfg), len(tags), _ptr(tags, _i64), _ptr(coords),
                                     len(elems), _ptr(elems, _i64), C.byref(h), err, len(err))
        else:
            donors = np.ascontiguousarray(part_boundary[0], dtype=np.int32)
            basis = np.ascontiguousarray(part_boundary[1], dtype=np.float64)
            rc = lib.wasl_gpu_create_part(
                C.byref(cfg), len(tags), _ptr(tags, _i64), _ptr(coords), len(elems),
                _ptr(elems, _i64), donors.shape[0] if donors.ndim else 0,
                donors.ctypes.data_as(C.POINTER(C.c_int32)), _ptr(basis), C.byref(h), err,
                len(err))
        self.part = part_boundary is not None
        if rc != 0:
            raise WaslError(rc, err.value.decode())
        self._lib, self._h = lib, h
        ne, nf = C.c_int64(), C.c_int64()
        nm, nv = C.c_int(), C.c_int()
        lib.wasl_gpu_sizes(h, C.byref(ne), C.byref(nf), C.byref(nm), C.byref(nv))
        self.elements, self.faces = ne.value, nf.value
        self.modes, self.variables = nm.value, nv.value
        self.state_size = self.elements * self.modes * self.variables

    def _check(self, rc):
        if rc != 0:
            raise WaslError(rc, self._lib.wasl_gpu_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.wasl_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- state ------------------------------------------------------------
    def set_state(self, coefficients):
        c = np.ascontiguousarray(coefficients, dtype=np.float64).ravel()
        self._check(self._lib.wasl_gpu_set_state(self._h, _ptr(c), c.size))

    def get_state(self) -> np.ndarray:
        c = np.empty(self.state_size)
        self._check(self._lib.wasl_gpu_get_state(self._h, _ptr(c), c.size))
        return c

    def get_state_into(self, out: np.ndarray):
        """Copy the state into a caller-owned contiguous float64 array (e.g. pinned)."""
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == self.state_size
        self._check(self._lib.wasl_gpu_get_state(self._h, _ptr(out), out.size))

    def vertices(self) -> np.ndarray:
        per = 6 if self.config.dimensions == 2 else 2
        v = np.empty(self.elements * per)
        self._check(self._lib.wasl_gpu_element_vertices(self._h, _ptr(v), v.size))
        return v.reshape(self.elements, per)

    # ---- quadrature, projection, evaluation ------------------------------------
    def rule_points(self, rule_order: int) -> int:
        n = C.c_int()
        self._check(self._lib.wasl_gpu_rule_points(self._h, rule_order, C.byref(n)))
        return n.value

    def quadrature(self, rule_order: int):
        """Physical points and weights [element][point]: (x, y, w) (y None in 1D)."""
        Q = self.rule_points(rule_order)
        x, w = np.empty((self.elements, Q)), np.empty((self.elements, Q))
        y = np.empty((self.elements, Q)) if self.config.dimensions == 2 else None
        self._check(self._lib.wasl_gpu_quadrature(self._h, rule_order, _ptr(x),
                                                  _ptr(y) if y is not None else None, _ptr(w)))
        return x, y, w

    def project(self, rule_order: int, values):
        """Set the state to the L2 projection of values [element][point][variable]."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self._lib.wasl_gpu_project(self._h, rule_order, _ptr(v), v.size))

    def evaluate(self, rule_order: int) -> np.ndarray:
        Q = self.rule_points(rule_order)
        v = np.empty((self.elements, Q, self.variables))
        self._check(self._lib.wasl_gpu_evaluate(self._h, rule_order, _ptr(v), v.size))
        return v

    # ---- stepping -----------------------------------------------------------
    def stable_dt(self, cfl: float) -> float:
        dt = C.c_double()
        self._check(self._lib.wasl_gpu_stable_dt(self._h, cfl, C.byref(dt)))
        return dt.value

    def cfl_parts(self):
        """(largest cell-average wave speed, smallest element length): the
        factors of stable_dt = cfl length / (speed (2p + 1)), for reductions
        over the ranks of a partitioned run (2D Euler)."""
        speed, length = C.c_double(), C.c_double()
        self._check(self._lib.wasl_gpu_cfl_parts(self._h, C.byref(speed), C.byref(length)))
        return speed.value, length.value

    def step(self, dt: float):
        self._check(self._lib.wasl_gpu_step(self._h, dt))

    def limit(self):
        """Apply the stage limiter to the current state (initial-state limiting)."""
        self._check(self._lib.wasl_gpu_limit(self._h))

    def run(self, cfl, start_time, end_time, max_steps=2**62):
        steps, time = C.c_uint64(), C.c_double()
        self._check(self._lib.wasl_gpu_run(self._h, cfl, start_time, end_time, max_steps,
                                           C.byref(steps), C.byref(time)))
        return steps.value, time.value

    def run_resident(self, cfl, start_time, end_time, max_steps=2**62):
        """run() in one kernel launch (small line meshes, no limiter)."""
        steps, time = C.c_uint64(), C.c_double()
        self._check(self._lib.wasl_gpu_run_resident(self._h, cfl, start_time, end_time,
                                                    max_steps, C.byref(steps), C.byref(time)))
        return steps.value, time.value

    def advance(self, cfl: float, steps: int, sync: bool = True):
        """Device-resident steps; with sync=False returns once they are
        enqueued (device errors then surface at sync())."""
        self._check(self._lib.wasl_gpu_advance(self._h, cfl, steps))
        if sync:
            self.sync()

    def sync(self):
        self._check(self._lib.wasl_gpu_sync(self._h))

    def flags(self) -> np.ndarray:
        f = np.empty(3 * self.elements, dtype=np.uint8)
        self._check(self._lib.wasl_gpu_get_flags(self._h, _ptr(f, _u8), f.size))
        return f.reshape(3, self.elements)

    def mass_energy(self):
        m, e = C.c_double(), C.c_double()
        self._check(self._lib.wasl_gpu_mass_energy(self._h, C.byref(m), C.byref(e)))
        return m.value, e.value

    # ---- device interop -------------------------------------------------------
    def element_order(self) -> np.ndarray:
        """order[i]: the caller's element stored at column i of the device state."""
        out = np.empty(self.elements, dtype=np.int64)
        self._check(self._lib.wasl_gpu_element_order(self._h, _ptr(out, _i64), out.size))
        return out

    def state_device_pointer(self) -> int:
        p = C.c_void_p()
        self._check(self._lib.wasl_gpu_state_device(self._h, C.byref(p)))
        return p.value

    def stream_handle(self) -> int:
        s = C.c_void_p()
        self._check(self._lib.wasl_gpu_stream(self._h, C.byref(s)))
        return s.value or 0

    # ---- setup products -----------------------------------------------------------
    SETUP_PHASES = ("topology", "order", "periodic", "faces", "stencil", "other")

    def setup_times(self) -> dict:
        """Wall-clock ms of each setup phase (wasl_gpu_setup_times)."""
        ms = np.zeros(len(self.SETUP_PHASES))
        self._check(self._lib.wasl_gpu_setup_times(self._h, _ptr(ms), len(ms)))
        return dict(zip(self.SETUP_PHASES, ms.tolist()))

    def stencil_transforms(self) -> np.ndarray:
        """The limiter's candidate transforms [element][3][target][source]."""
        out = np.empty((self.elements, 3, self.modes, self.modes))
        self._check(self._lib.wasl_gpu_stencil_transforms(self._h, _ptr(out), out.size))
        return out

    def periodic_trace(self, boundary_faces: int, points: int):
        """(donors [boundary face][point], basis [boundary face][point][mode])."""
        donors = np.empty((boundary_faces, points), dtype=np.int32)
        basis = np.empty((boundary_faces, points, self.modes))
        self._check(self._lib.wasl_gpu_periodic_trace(
            self._h, donors.ctypes.data_as(C.POINTER(C.c_int32)), _ptr(basis), donors.size))
        return donors, basis

    # ---- measurement ------------------------------------------------------------
    def tuning(self):
        """(kernel choice, per-variant stage ms) of the mixed form; see wasl_gpu_tuning."""
        choice, count = C.c_int(), C.c_int()
        ms = np.zeros(64)
        self._check(self._lib.wasl_gpu_tuning(self._h, C.byref(choice), _ptr(ms), len(ms),
                                              C.byref(count)))
        return choice.value, ms[:count.value].tolist()

    # ---- learned troubled-cell indicator -------------------------------------------

    def indicator_features(self) -> int:
        n = C.c_int()
        self._check(self._lib.wasl_gpu_indicator_features(self._h, C.byref(n)))
        return n.value

    def indicator_data(self):
        """(features [elements][F] float32, reference flags [elements] uint8) of
        the current state."""
        F = self.indicator_features()
        x = np.empty((self.elements, F), dtype=np.float32)
        y = np.empty(self.elements, dtype=np.uint8)
        self._check(self._lib.wasl_gpu_indicator_data(self._h, _ptr(x, _f), _ptr(y, _u8),
                                                      self.elements))
        return x, y

    def set_indicator(self, weights, lo=0.1, hi=0.9):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        self._check(self._lib.wasl_gpu_set_indicator(self._h, _ptr(w, _f), w.size, lo, hi))

    def set_indicator_kernel(self, kernel="tcgen05"):
        """The inference kernel: "tcgen05" (default) or "mma.sync"."""
        self._check(self._lib.wasl_gpu_indicator_kernel(
            self._h, {"tcgen05": 0, "mma.sync": 1}[kernel]))

    def indicator_logits(self):
        z = np.empty(self.elements, dtype=np.float32)
        self._check(self._lib.wasl_gpu_indicator_logits(self._h, _ptr(z, _f), self.elements))
        return z

    def indicator_stats(self, reset=False):
        """dict of cell-stage counts since set (or the last reset)."""
        s = (C.c_uint64 * 6)()
        self._check(self._lib.wasl_gpu_indicator_stats(self._h, s, 1 if reset else 0))
        keys = ["network_troubled", "network_smooth", "fallback", "reference_troubled",
                "missed", "false"]
        return dict(zip(keys, [int(v) for v in s]))

    def profile_begin(self):
        self._check(self._lib.wasl_gpu_profile_begin(self._h))

    def profile_end(self):
        """(summed stage-kernel ms, stage kernels timed, kernels launched)."""
        ms, k, n = C.c_double(), C.c_int64(), C.c_int64()
        self._check(self._lib.wasl_gpu_profile_end(self._h, C.byref(ms), C.byref(k), C.byref(n)))
        return ms.value, k.value, n.value

    def profile_stages(self):
        """The last profile_end's stage-kernel ms split by RK stage (0, 1, 2)."""
        out = np.zeros(3)
        self._check(self._lib.wasl_gpu_profile_stages(self._h, _ptr(out)))
        return out.tolist()

    # ---- restart files ----------------------------------------------------------
    def write_checkpoint(self, path, time, step, prepared_mesh=""):
        self._check(self._lib.wasl_gpu_write_checkpoint(self._h, os.fsencode(path), time, step,
                                                        os.fsencode(prepared_mesh)))

    def read_checkpoint(self, path):
        t, s = C.c_double(), C.c_uint64()
        self._check(self._lib.wasl_gpu_read_checkpoint(self._h, os.fsencode(path), C.byref(t),
                                                       C.byref(s)))
        return t.value, s.value


class Batch:
    """Many independent 2D Euler cases (triangle meshes, orders 1-3) advanced
    together in the mixed form (wasl_batch_* in include/wasl_b200.h).

    ``cases`` is a list of ``(node_tags, node_coordinates, element_nodes,
    polynomial_order)``.
    """

    def __init__(self, cases, *, gamma=1.4, boundary="transmissive", limiting=False,
                 sensor_threshold=1e-3, density_floor=1e-10, pressure_floor=1e-10,
                 reduced_volume_rule=True, tile_shape=0, use_graph=True, device=0,
                 positivity_all=False):
        lib = library()
        cfg = BatchConfig()
        lib.wasl_batch_config_default(C.byref(cfg))
        cfg.heat_capacity_ratio = gamma
        cfg.boundary = BOUNDARY_KINDS[boundary]
        cfg.limiting = 1 if limiting else 0
        cfg.sensor_threshold = sensor_threshold
        cfg.density_floor = density_floor
        cfg.pressure_floor = pressure_floor
        cfg.reduced_volume_rule = 1 if reduced_volume_rule else 0
        cfg.tile_shape = tile_shape
        cfg.use_graph = 1 if use_graph else 0
        cfg.device = device
        cfg.positivity_all = 1 if positivity_all else 0
        self.config = cfg
        orders = np.array([c[3] for c in cases], dtype=np.int32)
        node_counts = np.array([len(c[0]) for c in cases], dtype=np.int64)
        elem_counts = np.array([len(c[2]) for c in cases], dtype=np.int64)
        tags = np.ascontiguousarray(np.concatenate([np.asarray(c[0], np.int64) for c in cases]))
        xy = np.ascontiguousarray(np.concatenate([np.asarray(c[1], np.float64) for c in cases]))
        tris = np.ascontiguousarray(np.concatenate([np.asarray(c[2], np.int64) for c in cases]))
        err = C.create_string_buffer(1024)
        h = C.c_void_p()
        rc = lib.wasl_batch_create(C.byref(cfg), len(cases),
                                   orders.ctypes.data_as(C.POINTER(C.c_int)),
                                   _ptr(node_counts, _i64), _ptr(tags, _i64), _ptr(xy),
                                   _ptr(elem_counts, _i64), _ptr(tris, _i64), C.byref(h), err,
                                   len(err))
        if rc != 0:
            raise WaslError(rc, err.value.decode())
        self._lib, self._h = lib, h
        n, ne, dof = C.c_int64(), C.c_int64(), C.c_int64()
        self._check(lib.wasl_batch_sizes(h, C.byref(n), C.byref(ne), C.byref(dof)))
        self.cases, self.elements, self.dof = n.value, ne.value, dof.value
        self.orders = orders.tolist()

    def _check(self, rc):
        if rc != 0:
            raise WaslError(rc, self._lib.wasl_batch_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.wasl_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()

    def case_size(self, c):
        ne, nm = C.c_int64(), C.c_int()
        self._check(self._lib.wasl_batch_case_size(self._h, c, C.byref(ne), C.byref(nm)))
        return ne.value, nm.value

    def set_state(self, c, coefficients):
        a = np.ascontiguousarray(coefficients, dtype=np.float64).ravel()
        self._check(self._lib.wasl_batch_set_state(self._h, c, _ptr(a), a.size))

    def get_state(self, c):
        ne, nm = self.case_size(c)
        out = np.empty(4 * nm * ne)
        self._check(self._lib.wasl_batch_get_state(self._h, c, _ptr(out), out.size))
        return out

    def quadrature(self, c, rule_order):
        ne, _ = self.case_size(c)
        q = (rule_order + 1) ** 2
        x, y, w = (np.empty((ne, q)) for _ in range(3))
        self._check(self._lib.wasl_batch_quadrature(self._h, c, rule_order, _ptr(x), _ptr(y),
                                                    _ptr(w)))
        return x, y, w

    def project(self, c, rule_order, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self._lib.wasl_batch_project(self._h, c, rule_order, _ptr(a), a.size))

    def limit(self):
        """The stage limiter on every case's current state (as the reference
        limits the projected initial state)."""
        self._check(self._lib.wasl_batch_limit(self._h))

    def advance(self, cfl, steps):
        self._check(self._lib.wasl_batch_advance(self._h, cfl, steps))

    def times(self):
        t, dt = np.empty(self.cases), np.empty(self.cases)
        self._check(self._lib.wasl_batch_times(self._h, _ptr(t), _ptr(dt), self.cases))
        return t, dt

    def status(self):
        """Per case: 0, or 1 (non-physical average) / 2 (mean below a floor)
        for a case that failed and was frozen."""
        out = np.zeros(self.cases, dtype=np.int32)
        self._check(self._lib.wasl_batch_status(self._h, out.ctypes.data_as(C.POINTER(C.c_int)),
                                                self.cases))
        return out

    def tuning(self, polynomial_order):
        choice, count = C.c_int(), C.c_int()
        ms = np.zeros(64)
        self._check(self._lib.wasl_batch_tuning(self._h, polynomial_order, C.byref(choice),
                                                _ptr(ms), len(ms), C.byref(count)))
        return choice.value, ms[:count.value].tolist()

    def launches(self):
        per_step, graph, total = C.c_int64(), C.c_int(), C.c_int64()
        self._check(self._lib.wasl_batch_launches(self._h, C.byref(per_step), C.byref(graph),
                                                  C.byref(total)))
        return per_step.value, bool(graph.value), total.value

    def stream_handle(self) -> int:
        s = C.c_void_p()
        self._check(self._lib.wasl_batch_stream(self._h, C.byref(s)))
        return s.value or 0


class Mlp:
    """The indicator network on the GPU: training (wasl_mlp_*) with the
    project's own forward/backward and Adam kernels."""

    def __init__(self, features, seed=0, device=0):
        lib = library()
        err = C.create_string_buffer(512)
        h = C.c_void_p()
        rc = lib.wasl_mlp_create(features, seed, device, C.byref(h), err, len(err))
        if rc != 0:
            raise WaslError(rc, err.value.decode())
        self._lib, self._h, self.features = lib, h, features
        n = C.c_int64()
        self._check(lib.wasl_mlp_parameter_count(h, C.byref(n)))
        self.parameters = n.value

    def _check(self, rc):
        if rc != 0:
            raise WaslError(rc, self._lib.wasl_mlp_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.wasl_mlp_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()

    def set_data(self, features, labels):
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(labels, dtype=np.uint8)
        self._check(self._lib.wasl_mlp_set_data(self._h, _ptr(x, _f), _ptr(y, _u8), len(y)))

    def train(self, steps, batch=4096, learning_rate=1e-3, positive_weight=1.0):
        loss = C.c_double()
        self._check(self._lib.wasl_mlp_train(self._h, steps, batch, learning_rate,
                                             positive_weight, C.byref(loss)))
        return loss.value

    def gradient(self, features, labels, positive_weight=1.0):
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(labels, dtype=np.uint8)
        g = np.empty(self.parameters, dtype=np.float32)
        loss = C.c_double()
        self._check(self._lib.wasl_mlp_gradient(self._h, _ptr(x, _f), _ptr(y, _u8), len(y),
                                                positive_weight, _ptr(g, _f), C.byref(loss)))
        return g, loss.value

    def predict(self, features):
        x = np.ascontiguousarray(features, dtype=np.float32)
        z = np.empty(len(x), dtype=np.float32)
        self._check(self._lib.wasl_mlp_predict(self._h, _ptr(x, _f), len(x), _ptr(z, _f)))
        return z

    def weights(self):
        w = np.empty(self.parameters, dtype=np.float32)
        self._check(self._lib.wasl_mlp_get_weights(self._h, _ptr(w, _f), w.size))
        return w

    def set_weights(self, weights):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        self._check(self._lib.wasl_mlp_set_weights(self._h, _ptr(w, _f), w.size))
