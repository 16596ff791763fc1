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
    lib.wr_line_mesh_named_new.restype = C.c_void_p
    lib.wr_line_mesh_named_new.argtypes = lib.wr_line_mesh_new.argtypes
    lib.wr_run_scalar_advection_case.argtypes = SCALAR_ARGTYPES[:-2]
    lib.wr_run_euler_case.argtypes = EULER_ARGTYPES[:-2]
    lib.wr_inspect_checkpoint.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t]
    return lib


def twin_library():
    """libwasl_case_gpu.so: the C twins of the bridge's coarse functions."""
    if not os.path.exists(GPU_CASE):
        pytest.skip("oracle/_ref/libwasl_case_gpu.so not built")
    gpu = C.CDLL(GPU_CASE)
    gpu.wasl_run_euler_case_gpu.argtypes = EULER_ARGTYPES
    gpu.wasl_run_euler_case_gpu_ex.argtypes = EULER_ARGTYPES[:-4] + [C.c_int] + EULER_ARGTYPES[-4:]
    gpu.wasl_run_scalar_advection_case_gpu.argtypes = SCALAR_ARGTYPES
    text = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]
    gpu.wasl_inspect_checkpoint.argtypes = [C.c_char_p] + text
    gpu.wasl_inspect_prepared_mesh.argtypes = [C.c_char_p] + text
    gpu.wasl_export_checkpoint.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p] + text
    return gpu


_names = C.POINTER(C.c_char_p)
_u8 = C.POINTER(C.c_uint8)
# mesh, output, restart, limiting, threshold, floors, dimensions, p, gamma, cfl,
# t0, t1, max steps, intervals x3, kept checkpoints, regions (pointer, length),
# boundary names, kinds, values, count, summary (buffer, length)[, error]
EULER_ARGTYPES = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_double, C.c_double,
                  C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, _d, C.c_size_t,
                  _names, _u8, _d, C.c_size_t, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]
# mesh, output, restart, mpi, dimensions, p, velocity x/y, cfl, t0, t1, max
# steps, intervals x3, kept checkpoints, default, sine, amplitude, intervals,
# circles, boundaries, summary[, error]
SCALAR_ARGTYPES = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double,
                   C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_uint64,
                   C.c_uint64, C.c_uint64, C.c_uint64, C.c_double, C.c_int, C.c_double, _d,
                   C.c_size_t, _d, C.c_size_t, _names, _u8, _d, C.c_size_t, C.c_char_p,
                   C.c_size_t, C.c_char_p, C.c_size_t]


def boundaries(entries):
    """[(name, kind, value)] -> the bridge's three slices and their length."""
    n = len(entries)
    names = (C.c_char_p * max(n, 1))(*[e[0].encode() for e in entries])
    kinds = (C.c_uint8 * max(n, 1))(*[e[1] for e in entries])
    values = (C.c_double * max(n, 1))(*[e[2] for e in entries])
    return (C.cast(names, _names), C.cast(kinds, _u8), C.cast(values, _d), n)


def prepared_mesh(lib, path, dims, named=False):
    """The reference's own test meshes (a perturbed box or line), prepared;
    named: the line's ends carry the physical names "left" and "right"."""
    i64 = C.POINTER(C.c_int64)
    if dims == 2:
        tags, xy, cells = meshgen.irregular_box(6)
        new, write, free = lib.wr_tri_mesh_new, lib.wr_write_prepared_tri_mesh, lib.wr_tri_mesh_free
    else:
        tags, xy, cells = meshgen.irregular_line(16)
        new = lib.wr_line_mesh_named_new if named else lib.wr_line_mesh_new
        write, free = lib.wr_write_prepared_line_mesh, lib.wr_line_mesh_free
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


def run_reference(lib, mesh, out, p, limiting, dims=2, named=()):
    summary = C.create_string_buffer(1024)
    regions = REGIONS[dims]
    rc = lib.wr_run_euler_case(str(mesh).encode(), str(out).encode(), None,
                               *case_arguments(p, limiting, dims), regions.ctypes.data_as(_d),
                               regions.size, *boundaries(named), summary, len(summary))
    assert rc == 0, lib.wr_last_error()
    return summary.value.decode()


def run_twin(gpu, mesh, out, p, limiting, dims=2, named=(), precision=None):
    summary, err = C.create_string_buffer(1024), C.create_string_buffer(1024)
    regions = REGIONS[dims]
    args = (str(mesh).encode(), str(out).encode(), None, *case_arguments(p, limiting, dims),
            regions.ctypes.data_as(_d), regions.size, *boundaries(named))
    if precision is None:
        rc = gpu.wasl_run_euler_case_gpu(*args, summary, len(summary), err, len(err))
    else:
        rc = gpu.wasl_run_euler_case_gpu_ex(*args, precision, summary, len(summary), err,
                                            len(err))
    return rc, summary.value.decode(), err.value.decode()


def same_summary(a, b):
    """step= and time= equal; the checkpoint paths differ by run directory."""
    fa, fb = dict(x.split("=", 1) for x in a.split()), dict(x.split("=", 1) for x in b.split())
    return (fa["step"], fa["time"], os.path.basename(fa["checkpoint"])) == \
        (fb["step"], fb["time"], os.path.basename(fb["checkpoint"]))


def tree(directory):
    out = {}
    for name in sorted(os.listdir(directory)):
        with open(os.path.join(directory, name), "rb") as f:
            out[name] = f.read()
    return out


def test_reference_case_run_writes_its_run_directory(tmp_path):
    """The checker side on the CPU: the reference's run_euler_case from the
    bridge's arguments runs to t = 0.03 and writes history, snapshots and
    checkpoints."""
    lib = reference_library()
    mesh = tmp_path / "box.mesh"
    prepared_mesh(lib, mesh, 2)
    summary = run_reference(lib, mesh, tmp_path / "cpu", 2, True)
    fields = dict(x.split("=", 1) for x in summary.split())
    assert int(fields["step"]) > 4 and float(fields["time"]) == 0.03
    names = os.listdir(tmp_path / "cpu")
    assert "history.csv" in names and "solution.pvd" in names
    assert sum(n.startswith("checkpoint") for n in names) == 2


@pytest.mark.gpu
@pytest.mark.parametrize("dims,p,limiting,named", [
    (2, 1, False, ()), (2, 2, True, ()), (2, 3, True, ()), (1, 2, True, ()), (1, 1, False, ()),
    (1, 2, True, (("left", 2, 0.0), ("right", 2, 0.0))),
    (1, 1, False, (("left", 0, 0.0), ("right", 0, 0.0)))])
def test_reference_run_loop_drives_the_gpu_model(tmp_path, dims, p, limiting, named):
    """The twin of run_euler_case with the bridge's arguments (named
    boundaries included: periodic, or outflow line ends) writes the reference's
    run directory byte for byte and returns its summary."""
    lib, gpu = reference_library(), twin_library()
    mesh = tmp_path / "case.mesh"
    prepared_mesh(lib, mesh, dims, named=bool(named))
    cpu = run_reference(lib, mesh, tmp_path / "cpu", p, limiting, dims, named)
    rc, summary, err = run_twin(gpu, mesh, tmp_path / "gpu", p, limiting, dims, named)
    assert rc == 0, err
    assert same_summary(summary, cpu)
    a, b = tree(tmp_path / "cpu"), tree(tmp_path / "gpu")
    assert list(a) == list(b)
    for name in a:
        assert a[name] == b[name], name


@pytest.mark.gpu
def test_euler_twin_ex_runs_the_mixed_form(tmp_path):
    """wasl_run_euler_case_gpu_ex takes the precision form; the plain form is
    the drop-in, the mixed form runs the same case to the same end time."""
    lib, gpu = reference_library(), twin_library()
    mesh = tmp_path / "case.mesh"
    prepared_mesh(lib, mesh, 2)
    rc, plain, err = run_twin(gpu, mesh, tmp_path / "plain", 2, False, precision=0)
    assert rc == 0, err
    rc, mixed, err = run_twin(gpu, mesh, tmp_path / "mixed", 2, False, precision=1)
    assert rc == 0, err
    assert plain.split()[1] == mixed.split()[1] == "time=0.029999999999999999"


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


def scalar_call(fn, mesh, out, dims, p, mpi=0, named=(), error=True):
    summary, err = C.create_string_buffer(1024), C.create_string_buffer(1024)
    regions = (INTERVALS.ctypes.data_as(_d), INTERVALS.size, CIRCLES.ctypes.data_as(_d),
               CIRCLES.size)
    args = (str(mesh).encode(), str(out).encode(), None, mpi, *scalar_arguments(dims, p),
            *regions, *boundaries(named), summary, len(summary))
    rc = fn(*args, err, len(err)) if error else fn(*args)
    return rc, summary.value.decode(), err.value.decode()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,p,named", [
    (1, 2, ()), (1, 3, ()), (2, 1, ()), (2, 2, ()),
    (1, 2, (("left", 1, 0.5), ("right", 2, 0.0))),
    (1, 1, (("left", 1, -0.25), ("right", 2, 0.0)))])
def test_reference_run_loop_drives_the_gpu_scalar_model(tmp_path, dims, p, named):
    """The twin of run_scalar_advection_case (periodic, or an inflow value at
    the left end and outflow at the right) writes the reference's run
    directory byte for byte."""
    lib, gpu = reference_library(), twin_library()
    mesh = tmp_path / "case.mesh"
    prepared_mesh(lib, mesh, dims, named=bool(named))
    rc, cpu, _ = scalar_call(lib.wr_run_scalar_advection_case, mesh, tmp_path / "cpu", dims, p,
                             named=named, error=False)
    assert rc == 0, lib.wr_last_error()
    rc, summary, err = scalar_call(gpu.wasl_run_scalar_advection_case_gpu, mesh,
                                   tmp_path / "gpu", dims, p, named=named)
    assert rc == 0, err
    assert same_summary(summary, cpu)
    a, b = tree(tmp_path / "cpu"), tree(tmp_path / "gpu")
    assert list(a) == list(b)
    for name in a:
        assert a[name] == b[name], name


def test_twins_reject_bad_bridge_arguments_like_the_reference(tmp_path):
    """Argument errors come back as the reference bridge's messages, before
    any device work (so this runs without a GPU): an invalid boundary kind, a
    region slice of the wrong length, and MPI on a line mesh in a build
    without MPI (the reference's own message, from its run as well)."""
    lib, gpu = reference_library(), twin_library()
    mesh = tmp_path / "line.mesh"
    prepared_mesh(lib, mesh, 1, named=True)
    summary, err = C.create_string_buffer(256), C.create_string_buffer(256)
    bad_kind = boundaries((("left", 7, 0.0), ("right", 2, 0.0)))
    regions = REGIONS[1]
    rc = gpu.wasl_run_euler_case_gpu(str(mesh).encode(), str(tmp_path / "a").encode(), None,
                                     *case_arguments(1, False, 1), regions.ctypes.data_as(_d),
                                     regions.size, *bad_kind, summary, len(summary), err,
                                     len(err))
    assert rc == -2 and err.value == b"boundaries: invalid boundary kind"
    rc = gpu.wasl_run_euler_case_gpu(str(mesh).encode(), str(tmp_path / "a").encode(), None,
                                     *case_arguments(1, False, 1), regions.ctypes.data_as(_d),
                                     regions.size - 1, *boundaries(()), summary, len(summary),
                                     err, len(err))
    assert rc == -2 and err.value == b"initial.regions: invalid Euler region data"
    rc, _, message = scalar_call(gpu.wasl_run_scalar_advection_case_gpu, mesh, tmp_path / "b", 1,
                                 2, mpi=1)
    assert rc == -2 and message == "simulation: bridge was built without MPI support"
    rc, _, _ = scalar_call(lib.wr_run_scalar_advection_case, mesh, tmp_path / "c", 1, 2, mpi=1,
                           error=False)
    assert rc != 0 and lib.wr_last_error() == message.encode()


def test_checkpoint_and_mesh_utility_twins(tmp_path):
    """inspect_checkpoint, inspect_prepared_mesh and export_checkpoint twins
    on a run directory the reference wrote (host code, no GPU)."""
    lib, gpu = reference_library(), twin_library()
    mesh = tmp_path / "box.mesh"
    prepared_mesh(lib, mesh, 2)
    run_reference(lib, mesh, tmp_path / "cpu", 2, False)
    checkpoint = sorted(n for n in os.listdir(tmp_path / "cpu") if n.startswith("checkpoint"))[-1]
    path = str(tmp_path / "cpu" / checkpoint).encode()
    summary, err = C.create_string_buffer(512), C.create_string_buffer(512)
    assert gpu.wasl_inspect_checkpoint(path, summary, len(summary), err, len(err)) == 0
    expected = C.create_string_buffer(512)
    assert lib.wr_inspect_checkpoint(path, expected, len(expected)) == 0
    assert summary.value == expected.value and b"modes=6 elements=" in summary.value
    assert gpu.wasl_inspect_prepared_mesh(str(mesh).encode(), summary, len(summary), err,
                                          len(err)) == 0
    assert summary.value == b"2D mesh with 72 elements"
    out = tmp_path / "averages.vtu"
    assert gpu.wasl_export_checkpoint(path, str(mesh).encode(), str(out).encode(), summary,
                                      len(summary), err, len(err)) == 0, err.value
    assert summary.value == b"exported 72 cells" and out.stat().st_size > 0
    rc = gpu.wasl_inspect_checkpoint(str(tmp_path / "none.h5").encode(), summary, len(summary),
                                     err, len(err))
    assert rc == -2 and b"does not exist" in err.value


def test_case_twins_report_no_device_as_a_status(tmp_path):
    """Without a usable GPU the case twins return a status and a message, as
    the handle's entry points do, instead of failing the process."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib, gpu = reference_library(), twin_library()
    mesh = tmp_path / "case.mesh"
    prepared_mesh(lib, mesh, 2)
    rc, _, err = run_twin(gpu, mesh, tmp_path / "gpu", 2, True)
    assert rc == -2 and err
