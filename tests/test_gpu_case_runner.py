"""The reference's own run loop (run_serial_case: CFL stepping, history, VTU
snapshots, checkpoint rotation) with the GPU-backed case model
(wasl_b200/integration/serial_case_model.cpp) writes the same run directory,
byte for byte, as the reference's run_euler_case with its CPU model.

Both runs go through oracle/_ref: libwaslref.so is the reference's code (with
the binary stand-in for its HDF5 files) and libwasl_case_gpu.so the adapter
linked against it and libwasl_b200.so."""
import ctypes as C
import os

import numpy as np
import pytest

import pyoracle
from wasl_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPU_CASE = os.path.join(ROOT, "oracle", "_ref", "libwasl_case_gpu.so")
_d, _u64 = C.POINTER(C.c_double), C.POINTER(C.c_uint64)

# A uniform state with a denser, slower disc (shape 2 = circle) or interval
# (shape 1): the reference case regression's kind of initial data.
REGIONS = {2: np.array([[0, 0, 0, 0, 0, 0, 1.0, 0.4, -0.3, 1.0],
                        [2, 0, 0, 0.5, 0.5, 0.22, 1.6, 0.1, 0.2, 1.8]], dtype=np.float64),
           1: np.array([[0, 0, 0, 0, 0, 0, 1.0, 0.4, 0.0, 1.0],
                        [1, 0.3, 0.6, 0, 0, 0, 0.3, 0.0, 0.0, 0.2]], dtype=np.float64)}


def reference_library():
    if not pyoracle.Reference.available():
        pytest.skip("reference checker oracle/_ref not built")
    lib = pyoracle.Reference().lib
    lib.wr_write_prepared_tri_mesh.argtypes = [C.c_void_p, C.c_char_p]
    lib.wr_write_prepared_line_mesh.argtypes = [C.c_void_p, C.c_char_p]
    lib.wr_run_scalar_advection_case.argtypes = [
        C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
        C.c_double, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
        C.c_double, C.c_int, C.c_double, _d, C.c_int64, _d, C.c_int64, _u64, _d]
    lib.wr_run_euler_case.argtypes = [
        C.c_char_p, C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
        C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64,
        C.c_uint64, C.c_uint64, _d, C.c_int64, _u64, _d]
    return lib


def prepared_mesh(lib, path, dims):
    """The reference's own test meshes (a perturbed box or line), prepared."""
    i64 = C.POINTER(C.c_int64)
    if dims == 2:
        tags, xy, cells = meshgen.irregular_box(6)
        new, write, free = lib.wr_tri_mesh_new, lib.wr_write_prepared_tri_mesh, lib.wr_tri_mesh_free
    else:
        tags, xy, cells = meshgen.irregular_line(16)
        new, write = lib.wr_line_mesh_new, lib.wr_write_prepared_line_mesh
        free = lib.wr_line_mesh_free
    handle = new(len(tags), tags.ctypes.data_as(i64), xy.ctypes.data_as(_d), len(cells),
                 cells.ctypes.data_as(i64))
    assert handle, lib.wr_last_error()
    try:
        assert write(handle, str(path).encode()) == 0, lib.wr_last_error()
    finally:
        free(handle)


def case_arguments(p, limiting, dims=2):
    # limiting, sensor threshold, floors, dimensions, p, gamma, cfl, t0, t1,
    # max steps, history / visualization / checkpoint intervals, kept checkpoints
    return (int(limiting), 1e-4, 1e-10, 1e-10, dims, p, 1.4, 0.2, 0.0, 0.03, 10000, 1, 4, 4, 2)


def run_reference(lib, mesh, out, p, limiting, dims=2):
    steps, time = C.c_uint64(), C.c_double()
    regions = REGIONS[dims]
    rc = lib.wr_run_euler_case(str(mesh).encode(), str(out).encode(),
                               *case_arguments(p, limiting, dims), regions.ctypes.data_as(_d),
                               len(regions), C.byref(steps), C.byref(time))
    assert rc == 0, lib.wr_last_error()
    return steps.value, time.value


def tree(directory):
    out = {}
    for name in sorted(os.listdir(directory)):
        with open(os.path.join(directory, name), "rb") as f:
            out[name] = f.read()
    return out


def test_reference_case_run_writes_its_run_directory(tmp_path):
    """The checker side on the CPU: the reference's run_euler_case from flat
    arguments runs to t = 0.03 and writes history, snapshots and checkpoints."""
    lib = reference_library()
    mesh = tmp_path / "box.mesh"
    prepared_mesh(lib, mesh, 2)
    steps, time = run_reference(lib, mesh, tmp_path / "cpu", 2, True)
    assert steps > 4 and time == 0.03
    names = os.listdir(tmp_path / "cpu")
    assert "history.csv" in names and "solution.pvd" in names
    assert sum(n.startswith("checkpoint") for n in names) == 2


@pytest.mark.gpu
@pytest.mark.parametrize("dims,p,limiting", [(2, 1, False), (2, 2, True), (2, 3, True),
                                             (1, 2, True), (1, 1, False)])
def test_reference_run_loop_drives_the_gpu_model(tmp_path, dims, p, limiting):
    lib = reference_library()
    if not os.path.exists(GPU_CASE):
        pytest.skip("oracle/_ref/libwasl_case_gpu.so not built")
    gpu = C.CDLL(GPU_CASE)
    gpu.wasl_run_euler_case_gpu.argtypes = [
        C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_double,
        C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64,
        C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, _d, C.c_size_t, C.c_int, _u64, _d,
        C.c_char_p, C.c_size_t]
    mesh = tmp_path / "case.mesh"
    prepared_mesh(lib, mesh, dims)
    cpu = run_reference(lib, mesh, tmp_path / "cpu", p, limiting, dims)
    steps, time = C.c_uint64(), C.c_double()
    err = C.create_string_buffer(512)
    regions = REGIONS[dims]
    rc = gpu.wasl_run_euler_case_gpu(str(mesh).encode(), str(tmp_path / "gpu").encode(), None,
                                     *case_arguments(p, limiting, dims),
                                     regions.ctypes.data_as(_d), len(regions), 0,
                                     C.byref(steps), C.byref(time), err, len(err))
    assert rc == 0, err.value.decode()
    assert (steps.value, time.value) == cpu
    a, b = tree(tmp_path / "cpu"), tree(tmp_path / "gpu")
    assert list(a) == list(b)
    for name in a:
        assert a[name] == b[name], name


# Scalar advection as the reference's case regression sets it up: a default
# value, an interval (lower, upper, value) and a circle (centre, radius,
# value); on lines also the sine start.
INTERVALS = np.array([[0.2, 0.55, 1.0]])
CIRCLES = np.array([[0.5, 0.4, 0.25, 2.0]])


def scalar_arguments(dims, p):
    # dimensions, p, velocity x, velocity y, cfl, t0, t1, max steps, history /
    # visualization / checkpoint intervals, kept checkpoints, default value,
    # sine start, sine amplitude
    return (dims, p, 0.7, -0.4 if dims == 2 else 0.0, 0.3, 0.0, 0.2, 10000, 3, 4, 5, 2, 0.25,
            int(dims == 1 and p == 2), 1.5)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,p", [(1, 2), (1, 3), (2, 1), (2, 2)])
def test_reference_run_loop_drives_the_gpu_scalar_model(tmp_path, dims, p):
    lib = reference_library()
    if not os.path.exists(GPU_CASE):
        pytest.skip("oracle/_ref/libwasl_case_gpu.so not built")
    gpu = C.CDLL(GPU_CASE)
    gpu.wasl_run_scalar_advection_case_gpu.argtypes = [
        C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double,
        C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
        C.c_uint64, C.c_double, C.c_int, C.c_double, _d, C.c_size_t, _d, C.c_size_t, _u64, _d,
        C.c_char_p, C.c_size_t]
    mesh = tmp_path / "case.mesh"
    prepared_mesh(lib, mesh, dims)
    args = scalar_arguments(dims, p)
    regions = (INTERVALS.ctypes.data_as(_d), len(INTERVALS), CIRCLES.ctypes.data_as(_d),
               len(CIRCLES))
    cpu_steps, cpu_time = C.c_uint64(), C.c_double()
    rc = lib.wr_run_scalar_advection_case(str(mesh).encode(), str(tmp_path / "cpu").encode(),
                                          *args, *regions, C.byref(cpu_steps),
                                          C.byref(cpu_time))
    assert rc == 0, lib.wr_last_error()
    steps, time = C.c_uint64(), C.c_double()
    err = C.create_string_buffer(512)
    rc = gpu.wasl_run_scalar_advection_case_gpu(str(mesh).encode(),
                                                str(tmp_path / "gpu").encode(), None, *args,
                                                *regions, C.byref(steps), C.byref(time), err,
                                                len(err))
    assert rc == 0, err.value.decode()
    assert (steps.value, time.value) == (cpu_steps.value, cpu_time.value)
    a, b = tree(tmp_path / "cpu"), tree(tmp_path / "gpu")
    assert list(a) == list(b)
    for name in a:
        assert a[name] == b[name], name


def test_case_twins_report_no_device_as_a_status(tmp_path):
    """Without a usable GPU the case twins return a status and a message, as
    the handle's entry points do, instead of failing the process."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = reference_library()
    if not os.path.exists(GPU_CASE):
        pytest.skip("oracle/_ref/libwasl_case_gpu.so not built")
    gpu = C.CDLL(GPU_CASE)
    mesh = tmp_path / "case.mesh"
    prepared_mesh(lib, mesh, 2)
    err = C.create_string_buffer(512)
    steps, time = C.c_uint64(), C.c_double()
    regions = REGIONS[2]
    gpu.wasl_run_euler_case_gpu.argtypes = [
        C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_double,
        C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64,
        C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, _d, C.c_size_t, C.c_int, _u64, _d,
        C.c_char_p, C.c_size_t]
    rc = gpu.wasl_run_euler_case_gpu(str(mesh).encode(), str(tmp_path / "gpu").encode(), None,
                                     *case_arguments(2, True), regions.ctypes.data_as(_d),
                                     len(regions), 0, C.byref(steps), C.byref(time), err,
                                     len(err))
    assert rc == -2 and err.value
