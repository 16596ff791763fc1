"""Regenerate the committed golden fixtures from the reference.

Run where the reference sources are present and the reference checker is
built, naming the reference checkout in REF:

    make -C oracle ref REF=<reference checkout>
    REF=<reference checkout> python tests/golden/make_golden.py

* case_regression.json -- the reference's stored case-regression metrics,
  parsed from cpp/tests/runtime/case_regression_reference.txt (29 runs: step,
  time, coefficient sum, coefficient L2, final mass).
* ref_vectors.npz -- outputs of the reference's own code (oracle/_ref) on
  seeded inputs over the 5x5 irregular box of that regression: the Euler
  residual for P0-P3, one limited SSP-RK3 step and its limiter flags, so the
  GPU tests can check against the reference where the reference is absent.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import pyoracle  # noqa: E402
from golden_cases import GAMMA  # noqa: E402
from wasl_b200 import meshgen  # noqa: E402

REF = os.environ.get("REF", "")


def seeded_state(ne, p, seed, amplitude=0.05):
    """Smooth-ish physical Euler state with energy in every mode."""
    M = (p + 1) * (p + 2) // 2
    rng = np.random.Generator(np.random.PCG64(seed))
    c = amplitude * rng.standard_normal((4, M, ne))
    s2 = np.sqrt(2.0)
    c[0, 0] = s2 * (1.0 + 0.2 * rng.uniform(-1, 1, ne))
    c[1, 0] = s2 * 0.3 * rng.uniform(-1, 1, ne)
    c[2, 0] = s2 * 0.3 * rng.uniform(-1, 1, ne)
    c[3, 0] = s2 * (2.5 + 0.3 * rng.uniform(-1, 1, ne))
    return c.ravel()


def main():
    if not os.path.isdir(os.path.join(REF, "cpp", "tests")):
        sys.exit("set REF to the reference checkout")
    rows = {}
    with open(os.path.join(REF, "cpp/tests/runtime/case_regression_reference.txt")) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            name, step, time, total, l2, mass = line.split()
            rows[name] = dict(step=int(step), time=float(time), coefficient_sum=float(total),
                              coefficient_l2=float(l2), final_mass=float(mass))
    with open(os.path.join(HERE, "case_regression.json"), "w") as f:
        json.dump(rows, f, indent=1, sort_keys=True)

    ref = pyoracle.Reference()
    box = meshgen.irregular_box(5)
    mesh = ref.tri_mesh(*box)
    out = {}
    for p in range(4):
        c = seeded_state(mesh.ne, p, 100 + p)
        donors, basis = mesh.periodic_trace(p)
        ext = mesh.periodic_exterior(p, donors, basis, c)
        out[f"state_p{p}"] = c
        out[f"residual_p{p}"] = mesh.euler_residual(GAMMA, p, c, ext)
        if p > 0:
            stencil = mesh.stencil(p, donors)
            stepped = c.copy()
            mesh.euler_step(GAMMA, p, 2e-3, stepped, donors, basis, stencil=stencil,
                            threshold=1e-3)
            out[f"limited_step_p{p}"] = stepped
    np.savez_compressed(os.path.join(HERE, "ref_vectors.npz"), **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
