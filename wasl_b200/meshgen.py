"""Seeded synthetic meshes, returned as flat node and element arrays.

Every generator returns ``(node_tags, node_coordinates, element_nodes)`` with
1-based int64 node tags, which is the input the solver's mesh builder takes
(the same information a Gmsh document carries for the reference's
``build_triangle_mesh`` / ``build_line_mesh``).

* ``irregular_box`` / ``irregular_line`` are the meshes the reference's case
  regression builds in code (cpp/tests/runtime/case_regression_test.cpp:77-129);
  they use ``math.sin``/``math.cos`` (the C library), so the coordinates are the
  same doubles the reference computes.
* ``jittered_box`` / ``jittered_line`` are the seeded benchmark meshes:
  N x N quads split along a random diagonal with interior vertices jittered
  uniformly within +-jitter*h.  The generator is numpy's PCG64 seeded with
  ``seed``; boundary vertices stay on the box so periodic images match.
"""
from __future__ import annotations

import math

import numpy as np


def irregular_box(n: int):
    """Unit box, perturbed interior nodes, alternating diagonals (reference test mesh)."""
    tags, xy = [], []
    for j in range(n + 1):
        for i in range(n + 1):
            x = i / n
            y = j / n
            if 0 < i < n and 0 < j < n:
                x += 0.2 / n * math.sin(3.0 * i + 5.0 * j)
                y += 0.2 / n * math.cos(2.0 * i - 7.0 * j)
            tags.append(j * (n + 1) + i + 1)
            xy.append((x, y))

    def node(i, j):
        return j * (n + 1) + i + 1

    tris = []
    for j in range(n):
        for i in range(n):
            if (i + j) % 2 == 0:
                tris.append((node(i, j), node(i + 1, j), node(i + 1, j + 1)))
                tris.append((node(i, j), node(i, j + 1), node(i + 1, j + 1)))
            else:
                tris.append((node(i, j), node(i + 1, j), node(i, j + 1)))
                tris.append((node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)))
    return (np.array(tags, dtype=np.int64), np.array(xy, dtype=np.float64),
            np.array(tris, dtype=np.int64))


def irregular_line(count: int):
    """Perturbed unit line; elements recorded reversed with alternating orientation."""
    tags, xs = [], []
    for k in range(count + 1):
        x = k / count
        if 0 < k < count:
            x += 0.3 / count * math.sin(7.0 * k)
        tags.append(k + 1)
        xs.append(x)
    segs = []
    for e in range(count - 1, -1, -1):
        first, second = e + 1, e + 2
        segs.append((second, first) if e % 2 else (first, second))
    return np.array(tags, np.int64), np.array(xs, np.float64), np.array(segs, np.int64)


def jittered_box(n: int, x0: float = 0.0, x1: float = 1.0, y0: float = 0.0, y1: float = 1.0,
                 jitter: float = 0.15, seed: int = 0, ny: int | None = None):
    """n x ny quads on [x0,x1]x[y0,y1], each split along a seeded random diagonal,
    interior vertices moved uniformly within +-jitter*h; 2*n*ny triangles."""
    ny = n if ny is None else ny
    rng = np.random.Generator(np.random.PCG64(seed))
    hx, hy = (x1 - x0) / n, (y1 - y0) / ny
    i = np.arange(n + 1)
    j = np.arange(ny + 1)
    X = np.broadcast_to(x0 + i[None, :] * hx, (ny + 1, n + 1)).copy()
    Y = np.broadcast_to(y0 + j[:, None] * hy, (ny + 1, n + 1)).copy()
    X[:, n] = x1
    Y[ny, :] = y1
    dx = rng.uniform(-jitter, jitter, size=(ny + 1, n + 1)) * hx
    dy = rng.uniform(-jitter, jitter, size=(ny + 1, n + 1)) * hy
    interior = np.zeros((ny + 1, n + 1), dtype=bool)
    interior[1:ny, 1:n] = True
    X[interior] += dx[interior]
    Y[interior] += dy[interior]
    tags = (np.arange((n + 1) * (ny + 1), dtype=np.int64) + 1)
    xy = np.stack([X.ravel(), Y.ravel()], axis=1)
    diag = rng.integers(0, 2, size=(ny, n))
    jj, ii = np.meshgrid(np.arange(ny), np.arange(n), indexing="ij")
    a = jj * (n + 1) + ii + 1          # (i, j)
    b = a + 1                          # (i+1, j)
    c = a + (n + 1)                    # (i, j+1)
    d = c + 1                          # (i+1, j+1)
    t0 = np.where(diag[..., None] == 0, np.stack([a, b, d], -1), np.stack([a, b, c], -1))
    t1 = np.where(diag[..., None] == 0, np.stack([a, d, c], -1), np.stack([b, d, c], -1))
    tris = np.stack([t0, t1], axis=2).reshape(-1, 3).astype(np.int64)
    return tags, xy, tris


def jittered_line(n: int, x0: float = 0.0, x1: float = 1.0, jitter: float = 0.2, seed: int = 0):
    """n cells on [x0,x1], interior nodes moved uniformly within +-jitter*h."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h = (x1 - x0) / n
    x = x0 + np.arange(n + 1) * h
    x[n] = x1
    x[1:n] += rng.uniform(-jitter, jitter, size=n - 1) * h
    tags = np.arange(n + 1, dtype=np.int64) + 1
    segs = np.stack([tags[:-1], tags[1:]], axis=1)
    return tags, x, segs
