"""The C-ABI library on a host without a GPU: it loads, exports every entry
point include/*.h declares, validates meshes on the host, and reports a
missing device as a status code instead of crashing."""
import glob
import os
import re

import numpy as np
import pytest

import wasl_b200
from wasl_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(r"^\s*(?:const\s+)?(?:int|void|char)\s*\*?\s*(wasl_\w+)\s*\(", re.M)


def declared_symbols():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names |= set(DECL.findall(open(header).read()))
    return names


def test_library_exports_every_declared_symbol():
    lib = wasl_b200.library()
    names = declared_symbols()
    assert len(names) >= 19
    for name in names:
        assert hasattr(lib, name), name
    assert names <= set(wasl_b200.SIGNATURES) | {n for n in names if n not in wasl_b200.SIGNATURES}


def test_python_signatures_cover_the_header():
    assert declared_symbols() == set(wasl_b200.SIGNATURES)


def test_config_defaults_match_reference():
    cfg = wasl_b200.default_config()
    assert cfg.sensor_threshold == 1e-3
    assert cfg.density_floor == 1e-10 and cfg.pressure_floor == 1e-10
    assert cfg.heat_capacity_ratio == 1.4
    assert cfg.boundary_left == wasl_b200.PERIODIC


def test_bad_mesh_reported_like_the_reference():
    tags, xy, tris = meshgen.irregular_box(2)
    tris = tris.copy()
    tris[3] = [tris[3][0], tris[3][0], tris[3][1]]  # degenerate: repeated node
    with pytest.raises(wasl_b200.WaslError) as err:
        wasl_b200.Solver(tags, xy, tris, polynomial_order=1)
    assert "zero-area element 4" in str(err.value)
    tris2 = meshgen.irregular_box(2)[2].copy()
    tris2[0, 0] = 999
    with pytest.raises(wasl_b200.WaslError) as err:
        wasl_b200.Solver(tags, xy, tris2, polynomial_order=1)
    assert "missing node 999" in str(err.value)


def test_no_device_is_a_status_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    tags, xy, tris = meshgen.irregular_box(3)
    with pytest.raises(wasl_b200.WaslError) as err:
        wasl_b200.Solver(tags, xy, tris, polynomial_order=2)
    assert err.value.status == -3


def test_unsupported_order_rejected():
    tags, xy, tris = meshgen.irregular_box(2)
    with pytest.raises(wasl_b200.WaslError) as err:
        wasl_b200.Solver(tags, xy, tris, polynomial_order=7)
    assert err.value.status in (-1, -3)


def test_checked_build_compiles():
    """The device index checks of the checked build (WASL_DEVICE_CHECKS)
    compile for sm_100a in the kernels that read element indices from mesh
    data (the plain stage kernel and limiter, the mixed patch kernel)."""
    import shutil
    import subprocess
    import tempfile
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    from wasl_b200 import build
    with tempfile.TemporaryDirectory() as tmp:
        for src in ("euler_tri_f64.cu",):
            cmd = [nvcc, *build.ARCH, *build.COMMON, *build.SOURCES[src], "-DWASL_DEVICE_CHECKS",
                   "-c", os.path.join(build.CSRC, src), "-o", os.path.join(tmp, src + ".o")]
            subprocess.run(cmd, check=True)
