"""CPU oracle of the learned troubled-cell indicator (test infrastructure).

A numpy restatement of the network the CUDA kernels in wasl_b200/csrc/mlp.cu
compute, used by the tests as the checker of the GPU forward pass, gradients
and features; nothing in the product calls it.  The network and its features
have no counterpart in the reference; the features read the reference's
modal layout (cpp/include/wasl/dg/modal_layout.hpp:16-57) and the labels are
its modal-decay sensor (cpp/src/limiting/euler_modal_limiter.cpp:18-24,
cpp/include/wasl/limiting/troubled_cell/modal_decay.hpp:23-33).

Network: x[F] -> 64 ReLU -> 64 ReLU -> logit; inputs, the first hidden layer
and every weight rounded to BF16 (round to nearest even), FP32 arithmetic;
loss w (softplus(z) - y z) with w = positive_weight for y = 1.
"""
import numpy as np

HIDDEN = 64


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    bits = a.view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32)


def shape(features):
    """Offsets of W1 [64][F], b1, W2 [64][64], b2, w3, b3 in the flat vector."""
    o = {}
    o["w1"] = 0
    o["b1"] = o["w1"] + HIDDEN * features
    o["w2"] = o["b1"] + HIDDEN
    o["b2"] = o["w2"] + HIDDEN * HIDDEN
    o["w3"] = o["b2"] + HIDDEN
    o["b3"] = o["w3"] + HIDDEN
    o["count"] = o["b3"] + 1
    return o


def unpack(params, features):
    o = shape(features)
    p = np.asarray(params, dtype=np.float32)
    W1 = p[o["w1"]:o["b1"]].reshape(HIDDEN, features)
    b1 = p[o["b1"]:o["w2"]]
    W2 = p[o["w2"]:o["b2"]].reshape(HIDDEN, HIDDEN)
    b2 = p[o["b2"]:o["w3"]]
    w3 = p[o["w3"]:o["b3"]]
    b3 = p[o["b3"]]
    return W1, b1, W2, b2, w3, b3


def forward(params, x, rounding=True):
    """Logits and the intermediate values of the network (BF16-rounded unless
    rounding is False, which the oracle's own finite-difference check uses)."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float32))
    x = np.asarray(x, dtype=np.float32)
    W1, b1, W2, b2, w3, b3 = unpack(params, x.shape[1])
    xr = r(x)
    a1 = xr.astype(np.float64) @ r(W1).T.astype(np.float64) + b1
    h1 = (r(np.maximum(a1, 0.0).astype(np.float32)).astype(np.float64) if rounding
          else np.maximum(a1, 0.0))
    a2 = h1 @ r(W2).T.astype(np.float64) + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ r(w3).astype(np.float64) + float(b3)
    return z, (xr.astype(np.float64), a1, h1, a2, h2)


def loss_and_gradient(params, x, y, positive_weight=1.0, rounding=True):
    """Mean weighted binary cross-entropy and its gradient (straight through
    the BF16 rounding), in the flat parameter layout."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float32))
    x = np.asarray(x, dtype=np.float32)
    y = np.asarray(y, dtype=np.float64)
    n, F = x.shape
    W1, b1, W2, b2, w3, b3 = unpack(params, F)
    z, (xr, a1, h1, a2, h2) = forward(params, x, rounding)
    w = np.where(y > 0, positive_weight, 1.0)
    softplus = np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))
    loss = np.sum(w * (softplus - y * z)) / n
    d3 = w * (1.0 / (1.0 + np.exp(-z)) - y) / n
    gw3 = h2.T @ d3
    gb3 = d3.sum()
    D2 = np.outer(d3, r(w3).astype(np.float64)) * (h2 > 0)
    gW2 = D2.T @ h1
    gb2 = D2.sum(axis=0)
    D1 = (D2 @ r(W2).astype(np.float64)) * (h1 > 0)
    gW1 = D1.T @ xr
    gb1 = D1.sum(axis=0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])


def features(state, M, neighbors, F):
    """Per element: density modes m >= 1 over the mean for the cell and its
    three stencil neighbours (zeros where absent), then neighbour mean / cell
    mean - 1, each clamped to [-8, 8], zero padded to F.  state is
    U[variable][mode][element] (flat or shaped)."""
    ne = neighbors.shape[0]
    rho = np.asarray(state, dtype=np.float64).reshape(4, M, ne)[0]
    out = np.zeros((ne, F), dtype=np.float32)
    c0 = rho[0]
    inv = np.where(c0 != 0.0, 1.0 / np.where(c0 != 0.0, c0, 1.0), 0.0)
    clamp = lambda v: np.clip(v.astype(np.float32), -8.0, 8.0)  # noqa: E731
    out[:, :M - 1] = clamp((rho[1:] * inv).T)
    for j in range(3):
        nb = neighbors[:, j]
        ok = nb >= 0
        nbs = np.where(ok, nb, 0)
        n0 = rho[0, nbs]
        ninv = np.where(n0 != 0.0, 1.0 / np.where(n0 != 0.0, n0, 1.0), 0.0)
        cols = clamp((rho[1:, nbs] * ninv).T)
        out[:, (j + 1) * (M - 1):(j + 2) * (M - 1)] = np.where(ok[:, None], cols, 0.0)
        out[:, 4 * (M - 1) + j] = np.where(ok, clamp(n0 * inv - 1.0), 0.0)
    return out
