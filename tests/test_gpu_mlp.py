"""The learned troubled-cell indicator's kernels against the CPU oracle
(oracle/mlp_oracle.py): training gradients, the FP32 prediction pass, the
tensor-core inference kernel, the features, and the fallback to the
reference sensor."""
import numpy as np
import pytest

import mlp_oracle
import wasl_b200
from golden.make_golden import seeded_state
from wasl_b200 import cases, meshgen

pytestmark = pytest.mark.gpu


def random_samples(seed, n, F, scale=2.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = (scale * rng.standard_normal((n, F))).astype(np.float32)
    y = (rng.uniform(size=n) < 0.25).astype(np.uint8)
    return x, y


@pytest.mark.parametrize("F", [16, 32, 48])
def test_gradient_matches_oracle(F):
    """Mean-loss gradient of the GPU forward/backward kernels (FP32 arithmetic
    with the BF16 rounding, atomic accumulation over blocks) against the
    oracle in float64: within 1e-3 in norm, the loss within 1e-5."""
    x, y = random_samples(F, 512, F)
    with wasl_b200.Mlp(F, seed=F) as net:
        w = net.weights()
        g, loss = net.gradient(x, y, positive_weight=3.0)
    loss_o, g_o = mlp_oracle.loss_and_gradient(w, x, y, 3.0)
    assert abs(loss - loss_o) <= 1e-5 * abs(loss_o)
    assert np.linalg.norm(g - g_o) <= 1e-3 * np.linalg.norm(g_o)
    o = mlp_oracle.shape(F)
    for a, b in (("w1", "b1"), ("w2", "b2"), ("w3", "b3")):
        part, ref = g[o[a]:o[b]], g_o[o[a]:o[b]]
        assert np.linalg.norm(part - ref) <= 2e-3 * np.linalg.norm(ref) + 1e-9


def test_predict_matches_oracle():
    x, _ = random_samples(5, 1000, 32)
    with wasl_b200.Mlp(32, seed=7) as net:
        z = net.predict(x)
        w = net.weights()
    z_o, _ = mlp_oracle.forward(w, x)
    assert np.max(np.abs(z - z_o) / (1.0 + np.abs(z_o))) <= 1e-3


def test_training_learns_a_separable_rule():
    rng = np.random.Generator(np.random.PCG64(9))
    x = rng.standard_normal((16384, 16)).astype(np.float32)
    y = (x[:, 0] + 0.5 * x[:, 1] ** 2 - 0.5 * x[:, 2] > 0.3).astype(np.uint8)
    with wasl_b200.Mlp(16, seed=1) as net:
        net.set_data(x, y)
        first = net.train(1, batch=1024, learning_rate=3e-3)
        last = net.train(600, batch=1024, learning_rate=3e-3)
        accuracy = np.mean((net.predict(x) > 0) == (y > 0))
    assert last < 0.3 * first
    assert accuracy > 0.95


@pytest.mark.parametrize("kernel", ["tcgen05", "mma.sync"])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_features_labels_and_inference_match_oracle(p, kernel, oracle):
    """Features and reference labels of a state, and each tensor-core
    inference kernel's logits (BF16 MMAs, FP32 accumulation: tcgen05 with
    TMEM accumulators, and warp-level mma.sync) against the oracle's network
    on the oracle's features."""
    arrays = meshgen.jittered_box(10, jitter=0.15, seed=p)
    with wasl_b200.Solver(*arrays, polynomial_order=p, limiting=True) as g:
        state = seeded_state(g.elements, p, 50 + p, amplitude=0.05)
        g.set_state(state)
        F = g.indicator_features()
        x, y = g.indicator_data()
        with wasl_b200.Mlp(F, seed=p) as net:
            w = net.weights()
        g.set_indicator(w, lo=0.1, hi=0.9)
        g.set_indicator_kernel(kernel)
        z = g.indicator_logits()
    mesh = oracle.tri_mesh(*arrays)
    donors, _ = mesh.periodic_trace(p)
    stencil = mesh.stencil(p, donors)
    M = (p + 1) * (p + 2) // 2
    x_o = mlp_oracle.features(state, M, stencil.neighbors, F)
    assert np.array_equal(x, x_o)
    rho = state.reshape(4, M, -1)[0]
    total = np.sum(rho * rho, axis=0)
    high = np.sum(rho[stencil.highest_degree_begin:] ** 2, axis=0)
    y_o = ~((total == 0) | (high / total <= 1e-3))
    assert np.array_equal(y.astype(bool), y_o)
    z_o, _ = mlp_oracle.forward(w, x_o)
    close = np.abs(z - z_o) <= 1e-3 * (1.0 + np.abs(z_o))
    assert close.mean() >= 0.99 and np.max(np.abs(z - z_o)) <= 0.05


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_fallback_band_reproduces_the_reference_sensor(precision):
    """With the band (lo, hi) = (-1, 2) every cell falls back to the
    reference sensor: states and flags bit-identical to the run without the
    network."""
    arrays = meshgen.jittered_box(16, jitter=0.15, seed=4)
    problem = cases.QuadrantRiemann(seed=3)
    out = []
    for learned in (False, True):
        with wasl_b200.Solver(*arrays, polynomial_order=2, precision=precision, limiting=True,
                              boundary="transmissive") as g:
            cases.project_initial(g, problem.conserved)
            if learned:
                with wasl_b200.Mlp(g.indicator_features(), seed=2) as net:
                    g.set_indicator(net.weights(), lo=-1.0, hi=2.0)
            for _ in range(5):
                g.step(g.stable_dt(0.1))
            out.append((g.get_state(), g.flags()))
            if learned:
                stats = g.indicator_stats()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert stats["fallback"] == 5 * 3 * len(arrays[2])
    assert stats["missed"] == 0 and stats["false"] == 0
    assert stats["reference_troubled"] > 0


def test_inference_kernels_agree_on_a_large_mesh():
    """The tcgen05 and mma.sync inference kernels on 65k elements (many
    persistent tiles per CTA): logits within FP32 accumulation-order rounding
    of each other, and the same decisions away from the band's edges."""
    arrays = meshgen.jittered_box(160, jitter=0.15, seed=9)
    with wasl_b200.Solver(*arrays, polynomial_order=3, limiting=True) as g:
        g.set_state(seeded_state(g.elements, 3, 77, amplitude=0.05))
        with wasl_b200.Mlp(g.indicator_features(), seed=3) as net:
            g.set_indicator(net.weights(), lo=0.1, hi=0.9)
        z = {}
        for kernel in ("tcgen05", "mma.sync"):
            g.set_indicator_kernel(kernel)
            z[kernel] = g.indicator_logits()
    a, b = z["tcgen05"], z["mma.sync"]
    assert np.all(np.isfinite(a)) and np.std(a) > 0
    assert np.max(np.abs(a - b)) <= 1e-2 * (1.0 + np.max(np.abs(b)))
    assert np.mean(np.abs(a - b) <= 1e-3 * (1.0 + np.abs(b))) >= 0.99
