"""The mixed-precision form: the plain FP64 path's discretization with FP32
only on high-mode perturbations, and optionally a lower-order collapsed volume
rule (order p..p+2; the reference's residual uses p+2).  Checked against the
plain path (tolerances stated per test), for free-stream preservation, and for
conservation."""
import numpy as np
import pytest

import wasl_b200
from golden.make_golden import seeded_state
from wasl_b200 import cases, meshgen

pytestmark = pytest.mark.gpu

# mixed_kernel: 1 face-centric kernels, 2 + s the fused tile kernel in shape s
# (s = 0..3 the tile kernel, 4..7 the shared-face tile kernel, 8..11 the patch
# kernel, 12..13 the patch kernel with its volume term on the tensor cores).
KERNELS = [1, 2, 3, 4, 5]
TILE_SHAPES = 16
SHARED_KERNELS = [6, 7, 8, 9]
PERSISTENT_KERNELS = [16, 17]
PATCH_KERNELS = [10, 11, 12, 13]
MMA_KERNELS = [14, 15]


def pair(arrays, p, **kw):
    return (wasl_b200.Solver(*arrays, polynomial_order=p, precision="plain", **kw),
            wasl_b200.Solver(*arrays, polynomial_order=p, precision="mixed", **kw))


@pytest.mark.parametrize("p,rule", [(p, r) for p in (1, 2, 3) for r in (0, p, p + 1, -1)])
def test_uniform_flow_stays_uniform(p, rule):
    """A constant state is preserved to FP64 round-off: the FP32 part sees dU = 0."""
    arrays = meshgen.jittered_box(16, jitter=0.15, seed=p)
    plain, mixed = pair(arrays, p, volume_rule_order=rule)
    with plain, mixed:
        state = np.zeros((4, mixed.modes, mixed.elements))
        state[:, 0] = np.sqrt(2) * np.array([1.0, 0.3, -0.2, 2.6])[:, None]
        mixed.set_state(state.ravel())
        for _ in range(20):
            mixed.step(mixed.stable_dt(0.2))
        out = mixed.get_state().reshape(state.shape)
    assert np.max(np.abs(out - state)) <= 2e-13


@pytest.mark.parametrize("p", [1, 2, 3])
def test_one_step_close_to_plain(p):
    """|mixed - plain| after one step, relative to the step's change: <= 1e-6."""
    arrays = meshgen.jittered_box(24, jitter=0.15, seed=10 + p)
    plain, mixed = pair(arrays, p)
    with plain, mixed:
        c = seeded_state(plain.elements, p, 31 + p, amplitude=0.02)
        plain.set_state(c)
        mixed.set_state(c)
        dt = plain.stable_dt(0.15)
        assert dt == mixed.stable_dt(0.15)
        plain.step(dt)
        mixed.step(dt)
        a, b = plain.get_state(), mixed.get_state()
    change = np.max(np.abs(a - c))
    assert np.max(np.abs(a - b)) <= 1e-6 * change


@pytest.mark.parametrize("p,rule,kernel", [(p, r, k) for p in (1, 2, 3) for r in (0, p)
                                           for k in (1, 2, 8, 10)] +
                         [(2, 2, k) for k in (3, 4, 5, 12)] +
                         [(p, -1, k) for p in (1, 2, 3) for k in (2, 11, 14)])
def test_mass_and_energy_conserved(p, rule, kernel):
    """Periodic faces paired, interior faces evaluated by both sides with the
    same instructions: totals conserved to FP64 round-off."""
    arrays = meshgen.jittered_box(16, jitter=0.15, seed=4)
    with wasl_b200.Solver(*arrays, polynomial_order=p, precision="mixed",
                          volume_rule_order=rule, mixed_kernel=kernel) as g:
        g.set_state(seeded_state(g.elements, p, 9, amplitude=0.02))
        m0, e0 = g.mass_energy()
        for _ in range(50):
            g.step(g.stable_dt(0.15))
        m1, e1 = g.mass_energy()
    assert abs(m1 - m0) <= 1e-13 * abs(m0)
    assert abs(e1 - e0) <= 1e-13 * abs(e0)


@pytest.mark.parametrize("p,rule", [(2, 0), (2, 2), (3, 3), (2, -1), (3, -1)])
def test_vortex_accuracy_matches_plain(p, rule):
    """Isentropic vortex on a 64x64-quad mesh to t=0.5: the mixed form's L1
    density error is within 1.5x of the plain FP64 path's."""
    vortex = cases.IsentropicVortex()
    arrays = cases.vortex_mesh(64, seed=7)
    errors = {}
    for form in ("plain", "mixed"):
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision=form,
                              volume_rule_order=rule if form == "mixed" else 0) as g:
            cases.project_initial(g, vortex.conserved)
            steps, t = g.run(0.15, 0.0, 0.5)
            errors[form] = cases.l1_density_error(g, lambda x, y: vortex.conserved(x, y, t))
    assert errors["mixed"] <= 1.5 * errors["plain"]


def test_rule_order_out_of_range_is_rejected():
    arrays = meshgen.jittered_box(4, jitter=0.1, seed=1)
    with pytest.raises(wasl_b200.WaslError, match="volume rule"):
        wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", volume_rule_order=5)


def test_limited_mixed_runs_quadrant_riemann():
    """Limiter and positivity on the mixed form: physical averages throughout."""
    arrays = meshgen.jittered_box(32, jitter=0.15, seed=3)
    problem = cases.QuadrantRiemann(seed=3)
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", limiting=True,
                          boundary="transmissive") as g:
        cases.project_initial(g, problem.conserved)
        g.limit()
        m0, _ = g.mass_energy()
        g.run(0.1, 0.0, 0.05)
        flags = g.flags()
        state = g.get_state().reshape(4, g.modes, g.elements)
    assert flags.sum() > 0
    assert np.all(state[0, 0] > 0)


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kernel", [2, 3, 4, 5])
@pytest.mark.parametrize("boundary", ["periodic", "transmissive"])
def test_tile_kernel_matches_face_centric(p, kernel, boundary):
    """The fused tile kernel computes the face-centric form's arithmetic (up
    to FP32 contraction order): after three steps the states differ by at most
    1e-6 of the change the steps made."""
    arrays = meshgen.jittered_box(20, jitter=0.15, seed=20 + p)
    c = seeded_state(2 * 20 * 20, p, 40 + p, amplitude=0.02)
    out = {}
    for k in (1, kernel):
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision="mixed", mixed_kernel=k,
                              boundary=boundary) as g:
            g.set_state(c)
            for _ in range(3):
                g.step(g.stable_dt(0.15))
            out[k] = g.get_state()
            assert g.tuning()[0] == k - 1
    change = np.max(np.abs(out[1] - c))
    assert np.max(np.abs(out[kernel] - out[1])) <= 1e-6 * change


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("limiting", [False, True])
@pytest.mark.parametrize("boundary", ["periodic", "transmissive"])
def test_shared_face_kernel_is_bit_identical(p, limiting, boundary):
    """The shared-face tile kernel evaluates a face inside a tile once instead
    of once per element, with the same arithmetic, and the persistent tile
    kernel loops its resident CTAs over the tiles: every launch shape gives
    the tile kernel's states bit for bit, with and without the limiter (whose
    rough pass takes the elements next to jumps of the means)."""
    arrays = meshgen.jittered_box(20, jitter=0.15, seed=50 + p)
    c = seeded_state(2 * 20 * 20, p, 70 + p, amplitude=0.02)
    out = {}
    for k in [2] + SHARED_KERNELS + PERSISTENT_KERNELS:
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision="mixed", mixed_kernel=k,
                              boundary=boundary, limiting=limiting,
                              positivity_all=limiting) as g:
            g.set_state(c)
            for _ in range(4):
                g.step(g.stable_dt(0.1))
            out[k] = (g.get_state(), g.flags())
            assert g.tuning()[0] == k - 1
    assert np.max(np.abs(out[2][0] - c)) > 0
    for k in SHARED_KERNELS + PERSISTENT_KERNELS:
        assert np.array_equal(out[k][0], out[2][0]), f"kernel {k}"
        assert np.array_equal(out[k][1], out[2][1]), f"kernel {k}"


def test_uniform_flow_tile_transmissive():
    arrays = meshgen.jittered_box(12, jitter=0.15, seed=5)
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", mixed_kernel=2,
                          boundary="transmissive") as g:
        state = np.zeros((4, g.modes, g.elements))
        state[:, 0] = np.sqrt(2) * np.array([0.8, -0.2, 0.5, 2.0])[:, None]
        g.set_state(state.ravel())
        for _ in range(10):
            g.step(g.stable_dt(0.2))
        out = g.get_state().reshape(state.shape)
    assert np.max(np.abs(out - state)) <= 2e-13


def test_autotuner_times_every_variant():
    """mixed_kernel 0: the first step times the face-centric kernels and every
    tile shape and keeps the fastest; later solvers of the same class reuse it."""
    arrays = cases.vortex_mesh(32, seed=3)
    vortex = cases.IsentropicVortex()
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed") as g:
        assert g.tuning()[0] == -1
        cases.project_initial(g, vortex.conserved)
        g.step(g.stable_dt(0.15))
        choice, ms = g.tuning()
    assert len(ms) == 1 + TILE_SHAPES and all(t > 0 for t in ms)
    assert 0 <= choice < 1 + TILE_SHAPES and ms[choice] == min(ms)
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed") as g:
        cases.project_initial(g, vortex.conserved)
        g.step(g.stable_dt(0.15))
        assert g.tuning() == (choice, ms)


@pytest.mark.parametrize("kernel", [1, 2, 5])
def test_fused_cfl_speed_matches_cfl_kernels(kernel):
    """advance() with the tile kernel reduces the next step's CFL speed inside
    the last stage; the trajectory is bit-identical to one whose every dt comes
    from the standalone CFL kernels (set_state in between forces them)."""
    arrays = cases.vortex_mesh(24, seed=5)
    vortex = cases.IsentropicVortex()
    out = []
    for fused in (True, False):
        with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed",
                              mixed_kernel=kernel) as g:
            cases.project_initial(g, vortex.conserved)
            if fused:
                g.advance(0.15, 6)
            else:
                for _ in range(6):
                    g.advance(0.15, 1)
                    g.set_state(g.get_state())
            out.append(g.get_state())
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("p", [1, 2, 3])
def test_rough_pass_conserves_with_the_limiter(p):
    """With the limiter on, elements next to jumps of the means go to the
    tile kernel's second pass (FP64 faces at the jumps, FP32 elsewhere); the
    limiter keeps every cell average.  Periodic totals are conserved to FP64
    round-off, so both elements of every face still apply the same flux."""
    arrays = meshgen.jittered_box(16, jitter=0.15, seed=30 + p)
    with wasl_b200.Solver(*arrays, polynomial_order=p, precision="mixed", limiting=True,
                          mixed_kernel=2, positivity_all=True) as g:
        c = seeded_state(g.elements, p, 60 + p, amplitude=0.02)  # means jump up to 40%
        g.set_state(c)
        m0, e0 = g.mass_energy()
        for _ in range(20):
            g.step(g.stable_dt(0.1))
        m1, e1 = g.mass_energy()
        assert g.flags().sum() > 0
    assert abs(m1 - m0) <= 1e-13 * abs(m0)
    assert abs(e1 - e0) <= 1e-13 * abs(e0)


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_advance_enqueues_and_sync_reports_errors(precision):
    """wasl_gpu_advance only enqueues; a device error from those steps (here a
    negative cell-average density made on the host) is reported by sync."""
    arrays = meshgen.jittered_box(8, jitter=0.15, seed=2)
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision=precision) as g:
        state = seeded_state(g.elements, 2, 3, amplitude=0.01).reshape(4, g.modes, g.elements)
        state[0, 0, 5] = -0.5
        g.set_state(state.ravel())
        g.advance(0.15, 1, sync=False)
        with pytest.raises(wasl_b200.WaslError, match="not physical") as err:
            g.sync()
        assert err.value.status == -4


def test_profile_splits_stage_time_by_rk_stage():
    """profile_stages: the stage-kernel time of the last profile split over
    the three SSP-RK3 stages adds up to the total."""
    arrays = cases.vortex_mesh(16, seed=2)
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", mixed_kernel=8) as g:
        cases.project_initial(g, cases.IsentropicVortex().conserved)
        g.profile_begin()
        g.advance(0.15, 3)
        ms, kernels, launches = g.profile_end()
        split = g.profile_stages()
    assert kernels == 9 and launches >= kernels and all(t > 0 for t in split)
    assert abs(sum(split) - ms) <= 1e-9 * ms


@pytest.mark.parametrize("form,p,rule", [("plain", 1, 0), ("plain", 2, 0), ("mixed", 2, 2),
                                         ("mixed", 2, -1)])
def test_vortex_convergence_rate(form, p, rule):
    """Isentropic vortex on 16, 32 and 64 quads per side to t = 0.5: the L1
    density error falls at a rate of at least p + 0.6 between the two finest
    meshes (the reference's vortex check,
    cpp/tests/dg/euler_triangle_residual_test.cpp:214-233)."""
    vortex = cases.IsentropicVortex()
    errors = []
    for n in (16, 32, 64):
        with wasl_b200.Solver(*cases.vortex_mesh(n, seed=7), polynomial_order=p, precision=form,
                              volume_rule_order=rule) as g:
            cases.project_initial(g, vortex.conserved)
            steps, t = g.run(0.15, 0.0, 0.5)
            errors.append(cases.l1_density_error(g, lambda x, y: vortex.conserved(x, y, t)))
    rate = np.log(errors[1] / errors[2]) / np.log(2.0)
    assert errors[0] > errors[1] > errors[2]
    assert rate >= p + 0.6, (errors, rate)


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("boundary", ["periodic", "transmissive"])
def test_patch_kernel_matches_face_centric(p, boundary):
    """The patch kernel (traces once per element, faces once per patch) is
    the face-centric form's arithmetic up to FP32 rounding order: after three
    steps the states differ by at most 1e-6 of the change the steps made; all
    its launch shapes agree bit for bit (a face computes the same bits whether
    it lies inside a patch or between two)."""
    arrays = meshgen.jittered_box(20, jitter=0.15, seed=80 + p)
    c = seeded_state(2 * 20 * 20, p, 90 + p, amplitude=0.02)
    out = {}
    for k in [1] + PATCH_KERNELS:
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision="mixed", mixed_kernel=k,
                              boundary=boundary) as g:
            g.set_state(c)
            for _ in range(3):
                g.step(g.stable_dt(0.15))
            out[k] = g.get_state()
            assert g.tuning()[0] == k - 1
    change = np.max(np.abs(out[1] - c))
    assert np.max(np.abs(out[10] - out[1])) <= 1e-6 * change
    for k in PATCH_KERNELS[1:]:
        assert np.array_equal(out[k], out[10]), f"kernel {k}"


def test_tensor_core_patch_kernel_needs_the_limiter_off():
    arrays = meshgen.jittered_box(6, jitter=0.1, seed=2)
    with pytest.raises(wasl_b200.WaslError, match="tensor-core volume"):
        wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", limiting=True,
                         mixed_kernel=MMA_KERNELS[0])


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("boundary", ["periodic", "transmissive"])
def test_patch_kernel_with_the_limiter(p, boundary):
    """With the limiter the patch kernel evaluates a face across a jump of
    the cell means in FP64 from both sides (the tile kernels' islands) and
    raises the sensor's flags.  On four-quadrant data it stays as close to
    the plain FP64 path as the tile kernel does (the limiter's nonlinear
    weights amplify FP32 rounding differences, so the two mixed kernels are
    compared through the FP64 run), every patch shape agrees bit for bit,
    and mass, momentum and energy stay conserved to FP64 round-off
    (periodic)."""
    arrays = meshgen.jittered_box(24, jitter=0.15, seed=110 + p)
    problem = cases.QuadrantRiemann(seed=3)
    out = {}
    for k in [0, 2, 10, 11, 12, 13]:
        precision = "plain" if k == 0 else "mixed"
        kw = {} if k == 0 else {"mixed_kernel": k}
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision=precision, boundary=boundary,
                              limiting=True, positivity_all=True, **kw) as g:
            cases.project_initial(g, problem.conserved)
            g.limit()
            m0, e0 = g.mass_energy()
            flagged = 0
            for _ in range(4):
                g.step(g.stable_dt(0.1))
                flagged += int(g.flags().sum())
            out[k] = g.get_state()
            m1, e1 = g.mass_energy()
            assert flagged > 0
            if k:
                assert g.tuning()[0] == k - 1
            if boundary == "periodic":
                assert abs(m1 - m0) <= 1e-13 * abs(m0) and abs(e1 - e0) <= 1e-13 * abs(e0)
    tile = np.abs(out[2] - out[0])
    patch = np.abs(out[10] - out[0])
    assert np.mean(patch) <= 1.5 * np.mean(tile) + 1e-12
    assert np.max(patch) <= 3.0 * np.max(tile) + 1e-12
    for k in (11, 12, 13):
        assert np.array_equal(out[k], out[10]), f"kernel {k}"


def test_autotuner_includes_the_patch_kernel_with_the_limiter():
    arrays = cases.vortex_mesh(24, seed=3)
    vortex = cases.IsentropicVortex()
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", limiting=True) as g:
        cases.project_initial(g, vortex.conserved)
        g.step(g.stable_dt(0.15))
        choice, ms = g.tuning()
    assert ms[0] == 0.0  # the face-centric kernels have no FP64 islands
    assert all(ms[1 + sh] > 0 for sh in range(12))
    assert ms[1 + 12] == 0.0 and ms[1 + 13] == 0.0  # tensor-core volume: no limiter
    assert all(ms[1 + sh] > 0 for sh in (14, 15))


@pytest.mark.parametrize("kernel,limiting", [(1, False), (2, False), (8, False), (10, False),
                                             (2, True), (8, True)])
def test_storage_order_is_a_relabelling(kernel, limiting):
    """The mixed form stores its elements along a Morton curve (element_order
    "curve", the default): a relabelling only, so the states, flag sets and
    time steps match storage in the caller's order bit for bit."""
    arrays = meshgen.jittered_box(20, jitter=0.15, seed=12)
    c = seeded_state(2 * 20 * 20, 2, 13, amplitude=0.02)
    out = {}
    for order in ("caller", "curve"):
        with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed", mixed_kernel=kernel,
                              limiting=limiting, positivity_all=limiting,
                              element_order=order) as g:
            stored = g.element_order()
            assert sorted(stored) == list(range(g.elements))
            assert (order == "caller") == np.array_equal(stored, np.arange(g.elements))
            g.set_state(c)
            dts = []
            for _ in range(3):
                dts.append(g.stable_dt(0.1))
                g.step(dts[-1])
            out[order] = (g.get_state(), g.flags(), dts, g.mass_energy())
    a, b = out["caller"], out["curve"]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    assert np.allclose(a[3], b[3], rtol=1e-14, atol=0.0)


@pytest.mark.parametrize("p,rule", [(1, -1), (2, -1), (3, -1), (2, 2), (3, 3)])
@pytest.mark.parametrize("boundary", ["periodic", "transmissive"])
def test_tensor_core_volume_matches_the_fma_pipe(p, rule, boundary):
    """The patch kernel with its volume contractions as split-TF32 tensor-core
    products (FP32 accumulation) against the same kernel on the FMA pipe:
    after three steps the states differ by at most 1e-6 of the change the
    steps made, and its two launch shapes agree bit for bit."""
    arrays = meshgen.jittered_box(20, jitter=0.15, seed=60 + p)
    c = seeded_state(2 * 20 * 20, p, 61 + p, amplitude=0.02)
    out = {}
    for k in [10] + MMA_KERNELS:
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision="mixed", mixed_kernel=k,
                              boundary=boundary, volume_rule_order=rule) as g:
            g.set_state(c)
            for _ in range(3):
                g.step(g.stable_dt(0.15))
            out[k] = g.get_state()
    change = np.max(np.abs(out[10] - c))
    assert np.max(np.abs(out[14] - out[10])) <= 1e-6 * change
    assert np.array_equal(out[15], out[14])


@pytest.mark.parametrize("p", [2, 3])
def test_tensor_core_volume_vortex_accuracy(p):
    """Isentropic vortex, 64x64 quads to t = 0.5 with the tensor-core volume
    term: L1 density error within 1.5x of the plain FP64 path's."""
    vortex = cases.IsentropicVortex()
    arrays = cases.vortex_mesh(64, seed=7)
    errors = {}
    for form, kernel in (("plain", 0), ("mixed", 14)):
        with wasl_b200.Solver(*arrays, polynomial_order=p, precision=form, mixed_kernel=kernel,
                              volume_rule_order=-1 if form == "mixed" else 0) as g:
            cases.project_initial(g, vortex.conserved)
            steps, t = g.run(0.15, 0.0, 0.5)
            errors[form] = cases.l1_density_error(g, lambda x, y: vortex.conserved(x, y, t))
    assert errors["mixed"] <= 1.5 * errors["plain"]


@pytest.mark.parametrize("kernel", [11, 13])
def test_dependent_stage_launches_are_deterministic(kernel):
    """Each RK stage's patch kernel is launched as a programmatic dependent of
    the launch before it: its CTAs start while that launch drains and wait in
    hardware before reading the state.  Device-resident steps over a mesh of
    many CTA waves (131,072 triangles: 1,024 CTAs of 128) give the same bits
    on every run."""
    arrays = cases.vortex_mesh(256)
    vortex = cases.IsentropicVortex()
    runs = []
    with wasl_b200.Solver(*arrays, polynomial_order=2, precision="mixed",
                          mixed_kernel=kernel) as g:
        cases.project_initial(g, vortex.conserved)
        c = g.get_state()
        for _ in range(3):
            g.set_state(c)
            g.advance(0.15, 12)
            runs.append(g.get_state())
    assert not np.array_equal(runs[0], c)
    assert np.array_equal(runs[1], runs[0]) and np.array_equal(runs[2], runs[0])
