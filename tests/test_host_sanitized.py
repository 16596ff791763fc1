"""The host-side setup code (mesh topology, face slots, periodic pairing,
tile and patch arrays, the Morton order, limiter stencils, projection) built
with AddressSanitizer and UndefinedBehaviorSanitizer and run on seeded
meshes: no sanitizer finding and every consistency check of
tests/host_check.cpp holding.  CPU only."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from wasl_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "wasl_b200", "csrc")
CXX = shutil.which("g++")


@pytest.fixture(scope="module")
def host_check(tmp_path_factory):
    if CXX is None:
        pytest.skip("no g++")
    out = tmp_path_factory.mktemp("asan") / "host_check"
    cmd = [CXX, "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=undefined", "-fno-omit-frame-pointer",
           f"-I{CSRC}", f"-I{os.path.join(ROOT, 'include')}",
           os.path.join(ROOT, "tests", "host_check.cpp"), os.path.join(CSRC, "mesh.cpp"),
           os.path.join(CSRC, "tri_setup.cpp"), "-o", str(out), "-lpthread"]
    subprocess.run(cmd, check=True)
    return out


def write_mesh(path, tags, xy, tris):
    with open(path, "wb") as f:
        np.array([len(tags), len(tris)], dtype=np.int64).tofile(f)
        np.asarray(tags, dtype=np.int64).tofile(f)
        np.asarray(xy, dtype=np.float64).tofile(f)
        np.asarray(tris, dtype=np.int64).tofile(f)


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("periodic", [0, 1])
def test_host_setup_under_sanitizers(host_check, tmp_path, p, periodic):
    mesh = tmp_path / "mesh.bin"
    write_mesh(mesh, *meshgen.jittered_box(9, jitter=0.15, seed=p, ny=7))
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="print_stacktrace=1")
    run = subprocess.run([str(host_check), str(mesh), str(p), str(periodic)], env=env,
                         capture_output=True, text=True)
    assert run.returncode == 0, run.stderr[-4000:]
    assert "0 failures" in run.stdout
