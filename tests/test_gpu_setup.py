"""Mesh setup on the device against the oracle, bit for bit: the periodic
donor search with its donor basis, and the limiter stencil's candidate
transforms (built on the GPU with the C library's pow supplied by the host
for the powers whose rounding the device cannot settle).  Meshes: jittered,
irregular and regular (whose repeated point coordinates put many powers on
exact dyadic values), periodic and transmissive, with the caller's and the
curve element order."""
import numpy as np
import pytest

import wasl_b200
from wasl_b200 import meshgen

pytestmark = pytest.mark.gpu

MESHES = {
    "jittered": lambda: meshgen.jittered_box(24, jitter=0.15, seed=7, ny=19),
    "irregular": lambda: meshgen.irregular_box(9),
    "regular": lambda: meshgen.jittered_box(16, jitter=0.0, seed=0),
    "stretched": lambda: meshgen.jittered_box(20, x1=3.0, y0=-0.5, y1=0.25, jitter=0.2, seed=3),
}


def boundary_trace(om, p):
    """The oracle's periodic trace restricted to the boundary faces, in face
    order: donors [b][q], basis [b][q][mode]."""
    Q, M = p + 1, (p + 1) * (p + 2) // 2
    donors, basis = om.periodic_trace(p)
    faces = np.flatnonzero(om.face_right < 0)
    return (donors.reshape(om.nf, Q)[faces], basis.reshape(om.nf, Q, M)[faces])


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("mesh", sorted(MESHES))
@pytest.mark.parametrize("boundary", ["periodic", "transmissive"])
def test_stencil_transforms_match_the_oracle(oracle, p, mesh, boundary):
    arrays = MESHES[mesh]()
    om = oracle.tri_mesh(*arrays)
    donors = boundary_trace(om, p)[0] if boundary == "periodic" else None
    dense = om.periodic_trace(p)[0] if boundary == "periodic" else None
    expected = om.stencil(p, dense)
    for precision in ("plain", "mixed"):
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision=precision, limiting=True,
                              boundary=boundary) as g:
            got = g.stencil_transforms()
            assert np.array_equal(got, expected.transforms), (precision, donors is None)
            assert np.array_equal(np.signbit(got), np.signbit(expected.transforms))


@pytest.mark.parametrize("p", [0, 1, 2, 3])
@pytest.mark.parametrize("mesh", sorted(MESHES))
def test_periodic_trace_matches_the_oracle(oracle, p, mesh):
    arrays = MESHES[mesh]()
    om = oracle.tri_mesh(*arrays)
    donors, basis = boundary_trace(om, p)
    forms = ["plain", "mixed"] if p >= 1 else ["plain"]
    for precision in forms:
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision=precision,
                              boundary="periodic") as g:
            got_donors, got_basis = g.periodic_trace(*donors.shape)
            assert np.array_equal(got_donors, donors), precision
            assert np.array_equal(got_basis, basis), precision
    with wasl_b200.Solver(*arrays, equation="scalar_advection", polynomial_order=p,
                          velocity=(1.0, 0.5), boundary="periodic") as g:
        got_donors, got_basis = g.periodic_trace(*donors.shape)
        assert np.array_equal(got_donors, donors)
        assert np.array_equal(got_basis, basis)


def test_setup_times_are_reported():
    arrays = meshgen.jittered_box(32, jitter=0.15, seed=1)
    with wasl_b200.Solver(*arrays, polynomial_order=3, limiting=True, boundary="periodic") as g:
        t = g.setup_times()
    assert set(t) == set(wasl_b200.Solver.SETUP_PHASES)
    assert all(v >= 0.0 for v in t.values())
    assert t["topology"] > 0.0 and t["periodic"] > 0.0 and t["stencil"] > 0.0


def test_inspection_rejects_wrong_sizes():
    arrays = meshgen.jittered_box(8, jitter=0.15, seed=2)
    with wasl_b200.Solver(*arrays, polynomial_order=2, boundary="periodic") as g:
        with pytest.raises(wasl_b200.WaslError, match="no limiter"):
            g.stencil_transforms()
        with pytest.raises(wasl_b200.WaslError, match="boundary faces"):
            g.periodic_trace(3, 3)
    with wasl_b200.Solver(*arrays, polynomial_order=2, boundary="transmissive") as g:
        with pytest.raises(wasl_b200.WaslError, match="no periodic faces"):
            g.periodic_trace(1, 3)
