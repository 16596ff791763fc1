"""The library's triangle topology (mesh.cpp) against the oracle's, which is
pinned to the reference's mesh build: vertices after reorientation, node
tags, faces in (left element, left edge) order with their sides, local
edges, orientation flips and normals, on jittered meshes with dense,
sparse-and-shuffled and reversed numberings; and the reference's errors
for duplicate tags, missing nodes, zero-area elements and non-conforming
edges.  CPU only."""
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
def dump(tmp_path_factory):
    if CXX is None:
        pytest.skip("no g++")
    out = tmp_path_factory.mktemp("topology") / "topology_dump"
    subprocess.run([CXX, "-std=c++20", "-O2", "-ffp-contract=off", f"-I{CSRC}",
                    f"-I{os.path.join(ROOT, 'include')}",
                    os.path.join(ROOT, "tests", "topology_dump.cpp"),
                    os.path.join(CSRC, "mesh.cpp"), "-o", str(out), "-lpthread"], check=True)
    return out


def run(dump, tmp_path, tags, xy, tris):
    mesh, out = tmp_path / "mesh.bin", tmp_path / "topology.bin"
    with open(mesh, "wb") as f:
        np.array([len(tags), len(tris)], dtype=np.int64).tofile(f)
        np.asarray(tags, dtype=np.int64).tofile(f)
        np.asarray(xy, dtype=np.float64).tofile(f)
        np.asarray(tris, dtype=np.int64).tofile(f)
    subprocess.run([str(dump), str(mesh), str(out)], check=True)
    raw = out.read_bytes()
    if raw.startswith(b"ERR "):
        return raw[4:].decode()
    ne, nf = np.frombuffer(raw[:16], dtype=np.int64)
    fields = [("vertices", np.float64, 6 * ne), ("nodes", np.int64, 3 * ne),
              ("face_left", np.int32, nf), ("face_right", np.int32, nf),
              ("face_left_edge", np.int32, nf), ("face_right_edge", np.int32, nf),
              ("face_flip", np.uint8, nf), ("face_nx", np.float64, nf),
              ("face_ny", np.float64, nf), ("face_scale", np.float64, nf)]
    at, topo = 16, {}
    for name, dtype, n in fields:
        size = np.dtype(dtype).itemsize * int(n)
        topo[name] = np.frombuffer(raw[at:at + size], dtype=dtype)
        at += size
    topo["vertices"] = topo["vertices"].reshape(ne, 6)
    topo["nodes"] = topo["nodes"].reshape(ne, 3)
    return topo


def numberings(n, seed):
    """The same jittered mesh with dense tags, with sparse shuffled tags and
    shuffled nodes, and with shuffled elements of mixed orientation."""
    rng = np.random.default_rng(seed)
    tags, xy, tris = (np.asarray(a) for a in meshgen.jittered_box(n, jitter=0.15, seed=seed))
    yield "dense", tags, xy, tris
    perm = rng.permutation(len(tags))
    sparse = tags * 7919 + 13
    lookup = dict(zip(tags.tolist(), sparse.tolist()))
    yield "sparse", sparse[perm], xy[perm], np.vectorize(lookup.get)(tris)
    shuffled = tris[rng.permutation(len(tris))].copy()
    flip = rng.random(len(shuffled)) < 0.5
    shuffled[flip] = shuffled[flip][:, [0, 2, 1]]
    yield "shuffled", tags, xy, shuffled


@pytest.mark.parametrize("n", [3, 16, 41])
def test_topology_matches_the_oracle(oracle, dump, tmp_path, n):
    for name, tags, xy, tris in numberings(n, seed=n):
        topo = run(dump, tmp_path, tags, xy, tris)
        om = oracle.tri_mesh(tags, xy, tris)
        assert np.array_equal(topo["vertices"], om.vertices), name
        assert np.array_equal(topo["nodes"], om.nodes), name
        for field in ("face_left", "face_right", "face_left_edge"):
            assert np.array_equal(topo[field], getattr(om, field)), (name, field)
        inner = om.face_right >= 0
        assert np.array_equal(topo["face_right_edge"][inner], om.face_right_edge[inner]), name
        flips = (om.face_left_v0 != om.face_right_v0)[inner]
        assert np.array_equal(topo["face_flip"][inner].astype(bool), flips), name
        assert np.array_equal(topo["face_nx"], om.face_normal_x), name
        assert np.array_equal(topo["face_ny"], om.face_normal_y), name


def test_topology_errors(dump, tmp_path):
    tags, xy, tris = (np.asarray(a) for a in meshgen.jittered_box(4, jitter=0.1, seed=1))
    dup = tags.copy()
    dup[5] = dup[3]
    assert run(dump, tmp_path, dup, xy, tris) == "triangle mesh: duplicate node tag 4"
    missing = tris.copy()
    missing[7, 1], missing[3, 2] = 99999, 88888
    assert (run(dump, tmp_path, tags, xy, missing) ==
            "triangle mesh: element references missing node 88888")
    zero = tris.copy()
    zero[9] = [zero[9][0], zero[9][0], zero[9][1]]
    assert run(dump, tmp_path, tags, xy, zero) == "triangle mesh: zero-area element 10"
    extra = np.vstack([tris, tris[[5, 2]]])
    message = run(dump, tmp_path, tags, xy, extra)
    # The repeated elements' interior edges now have three sides; the first
    # in (smaller tag, larger tag) order is reported.
    count = {}
    for t in extra.tolist():
        for i in range(3):
            edge = tuple(sorted((t[i], t[(i + 1) % 3])))
            count[edge] = count.get(edge, 0) + 1
    a, b = min(edge for edge, c in count.items() if c > 2)
    assert message == (f"triangle mesh: edge {a}-{b} has more than two adjacent elements"
                       " (non-conforming mesh)")
