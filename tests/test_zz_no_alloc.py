"""The allocation-free CFL entry point, checked against the handle's own.

wasl_cfl_dt_static serves callers that cannot call cudaMalloc (an
application whose device memory belongs to its own pool allocator, or a
latency-critical loop that cannot take cudaMalloc's implicit device
synchronization): it reduces a device-resident state with scratch held in a
fixed static device array.  Here it must give wasl_gpu_stable_dt's dt (the
same CFL rule, evaluated through a solver handle) bit for bit on two calls in
a row, with a step of the state in between.  This file is collected
last, so a failure here comes after every other test has run.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def test_static_scratch_cfl_matches_handle():
    import torch
    import pyoracle
    import wasl_b200
    from wasl_b200 import cases

    lib = wasl_b200.library()
    p, cfl = 2, 0.15
    arrays = cases.vortex_mesh(48, seed=5)
    length = pyoracle.Oracle().tri_mesh(*arrays).minimum_altitude()
    vortex = cases.IsentropicVortex()
    dt_device = torch.zeros(1, dtype=torch.float64, device="cuda")
    err = C.create_string_buffer(512)
    with wasl_b200.Solver(*arrays, polynomial_order=p) as g:
        cases.project_initial(g, vortex.conserved)
        for call in range(2):
            expected = g.stable_dt(cfl)
            rc = lib.wasl_cfl_dt_static(g.state_device_pointer(), g.elements, g.modes, 2, p,
                                        1.4, cfl, length, dt_device.data_ptr(),
                                        g.stream_handle(), err, len(err))
            assert rc == 0, err.value.decode()
            got = float(dt_device.item())
            assert got == expected, call
            g.step(expected)


def test_static_scratch_cfl_rejects_oversize_and_nonphysical():
    import torch
    import wasl_b200

    lib = wasl_b200.library()
    err = C.create_string_buffer(512)
    dt_device = torch.zeros(1, dtype=torch.float64, device="cuda")
    state = torch.zeros(4 * 8, dtype=torch.float64, device="cuda")
    rc = lib.wasl_cfl_dt_static(state.data_ptr(), 3_000_000_000, 1, 2, 0, 1.4, 0.1, 1.0,
                                dt_device.data_ptr(), None, err, len(err))
    assert rc == -1 and b"outside" in err.value
    rc = lib.wasl_cfl_dt_static(state.data_ptr(), 8, 1, 2, 0, 1.4, 0.1, 1.0,
                                dt_device.data_ptr(), None, err, len(err))
    assert rc == -4 and b"not physical" in err.value
    good = torch.tensor(np.sqrt(2) * np.repeat([1.0, 0.5, 0.0, 2.5], 8), dtype=torch.float64,
                        device="cuda")
    rc = lib.wasl_cfl_dt_static(good.data_ptr(), 8, 1, 2, 0, 1.4, 0.1, 1.0,
                                dt_device.data_ptr(), None, err, len(err))
    assert rc == 0
    speed = 0.5 + np.sqrt(1.4 * 0.4 * (2.5 - 0.125))
    assert float(dt_device.item()) == pytest.approx(0.1 / speed, rel=1e-14)
