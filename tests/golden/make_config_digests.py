"""Digests of the reference's own SSP-RK3 steps on the full benchmark meshes.

Run where the reference sources are present and its checker is built
(``make -C oracle ref REF=<reference checkout>``):

    python tests/golden/make_config_digests.py vortex256      # ~25 min, 1 core
    python tests/golden/make_config_digests.py quadrant1024   # ~15 min
    python tests/golden/make_config_digests.py shockvortex1024  # ~30 min

Each run writes ``tests/golden/digests_<name>.json``: the sha256 of the
initial coefficient vector, and for every step the reference's CFL time step
(``euler_cfl_timestep``, as a float hex string), the sha256 of the state after
the step (U[variable][mode][element], FP64 little-endian) and, for limited
runs, the sha256 of the three stages' troubled-cell flag sets (one byte per
element, stage after stage).  The states are far too large to commit (25 MB
to 1.3 GB); the digests let ``tests/test_gpu_config_parity.py`` check the GPU
plain path against the reference bit for bit on a box without the reference.

The inputs are built the same way on both sides, on the CPU: the seeded mesh
generator (``wasl_b200.meshgen``), the seeded initial data
(``wasl_b200.cases``) evaluated at the points of the order-max(p, 5) volume
rule, projected by the oracle's L2 projection (``wo_tri_project``), then, for
limited runs, one application of the reference limiter, as a case's first
state is limited before the first step.

* vortex256: the isentropic vortex on 256x256 jittered quads (131,072
  triangles), P2, periodic, limiter off, CFL 0.15, 100 steps.
* quadrant1024: the seeded four-quadrant Riemann problem on 1024x1024
  quads (2,097,152 triangles), P3, transmissive, limiter (WENO + positivity
  in troubled cells, as the reference limits), CFL 0.1, 2 steps.
* shockvortex1024: the Mach 1.1 shock-vortex on [0,2]x[0,1], 2048x1024 quads
  (4,194,304 triangles), P3, transmissive, limiter, CFL 0.1, 1 step.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from wasl_b200 import cases, meshgen  # noqa: E402

GAMMA = 1.4


def configs():
    """name -> (mesh arrays thunk, initial field, p, boundary, limiting, cfl, steps)."""
    return {
        "vortex256": (lambda: cases.vortex_mesh(256), cases.IsentropicVortex().conserved, 2,
                      "periodic", False, 0.15, 100),
        "quadrant1024": (lambda: meshgen.jittered_box(1024, jitter=0.15, seed=3),
                         cases.QuadrantRiemann(seed=3).conserved, 3, "transmissive", True, 0.1, 2),
        "shockvortex1024": (lambda: meshgen.jittered_box(2048, 0.0, 2.0, 0.0, 1.0, jitter=0.15,
                                                         seed=5, ny=1024),
                            cases.ShockVortex(seed=5).conserved, 3, "transmissive", True, 0.1, 1),
    }


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def initial_state(oracle, arrays, field, p):
    """The projected initial coefficients (oracle L2 projection, order
    max(p, 5) rule, the rule of cpp/src/case/initial_state.cpp:18-24)."""
    mesh = oracle.tri_mesh(*arrays)
    rule = max(p, 5)
    x, y = mesh.rule_points(rule)
    return mesh.project(p, rule, field(x, y))


def main(name):
    import pyoracle
    make_arrays, field, p, boundary, limiting, cfl, steps = configs()[name]
    t0 = time.time()
    arrays = make_arrays()
    c = initial_state(pyoracle.Oracle(), arrays, field, p)
    out = {"config": name, "polynomial_order": p, "boundary": boundary, "limiting": limiting,
           "cfl": cfl, "elements": int(len(arrays[2])), "initial_sha256": sha(c)}
    ref = pyoracle.Reference()
    mesh = ref.tri_mesh(*arrays)
    donors = basis = None
    if boundary == "periodic":
        donors, basis = mesh.periodic_trace(p)
    stencil = mesh.stencil(p, donors) if limiting else None
    print(f"{name}: setup {time.time() - t0:.0f} s", flush=True)
    if limiting:
        stencil.limit(GAMMA, 1e-3, 1e-10, 1e-10, c)
        out["limited_initial_sha256"] = sha(c)
    rows = []
    for k in range(steps):
        dt = mesh.cfl(GAMMA, c, p, cfl)
        flags = mesh.euler_step_ex(GAMMA, p, dt, c, boundary=boundary, donors=donors,
                                   basis=basis, stencil=stencil)
        row = {"dt": float(dt).hex(), "state_sha256": sha(c)}
        if limiting:
            row["flags_sha256"] = sha(flags)
            row["troubled"] = [int(s) for s in flags.sum(axis=1)]
        rows.append(row)
        print(f"{name}: step {k + 1} dt {dt:.6e} {time.time() - t0:.0f} s", flush=True)
    out["steps"] = rows
    with open(os.path.join(HERE, f"digests_{name}.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1])
