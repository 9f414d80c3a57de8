"""Writes the golden fixtures of tests/test_golden.py from micm itself.

micm's CPU Rosenbrock is compiled from the reference sources into
oracle/_ref/libmicm_ref.so (oracle/Makefile); this script runs it on small
seeded cases and stores its outputs.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from micm_b200 import synthetic  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def kernels(name, mech, n, seed, tableau=4):
    """Per-stage values: rate constants, forcing, -J, LU, linear solve, NormalizedError."""
    ref = oracle.Reference(mech, tableau=tableau)
    inp = synthetic.cell_inputs(mech, n, seed)
    k = ref.rate_constants(inp["temperature"], inp["pressure"], inp["air_density"], inp["custom_params"])
    y = ref.y_to_columns(inp["concentrations"])
    f = ref.forcing(k, y)
    j = ref.jacobian(k, y)
    a = j.copy()
    alpha = 1.0 / (30.0 * 0.5728200000000001)
    diag = [e for e, (r, c) in enumerate(zip(ref.rows, ref.cols)) if r == c]
    a[:, diag] += alpha
    lu = ref.decompose(a)
    x = ref.linear_solve(lu, f)
    ynew = y + 1e-3 * f
    err = 1e-4 * f
    ne = ref.normalized_error(y, ynew, err)
    np.savez_compressed(os.path.join(HERE, f"{name}_kernels.npz"), temperature=inp["temperature"],
                        pressure=inp["pressure"], air_density=inp["air_density"], custom_params=inp["custom_params"],
                        y=y, k=k, forcing=f, jacobian=j, alpha=alpha, lu=lu, x=x, ynew=ynew, err=err,
                        normalized_error=ne, rows=ref.rows, cols=ref.cols, species_columns=ref.species_columns)


def solves(name, mech, n, seed, tableau, dt, inputs_kw):
    """Per-cell solves: final concentrations (system order) and per-cell statistics."""
    ref = oracle.Reference(mech, tableau=tableau)
    inp = synthetic.cell_inputs(mech, n, seed, **inputs_kw)
    y, stats = ref.solve_per_cell(inp, dt, threads=1)
    np.savez_compressed(os.path.join(HERE, f"{name}_per_cell.npz"), y_final=y, stats=stats, dt=dt,
                        tableau=tableau, seed=seed, **inp)


def readme():
    """micm's README example (README.md:95-182) for 8 seeded cells, 10 global solves of 500 s."""
    mech = synthetic.readme_mechanism()
    ref = oracle.Reference(mech, tableau=3)
    inp = synthetic.cell_inputs(mech, 8, 11, readme_foo=(1.0, 30.0))
    ys = []
    cur = dict(inp)
    for _ in range(10):
        y, _ = ref.solve_global(cur, 500.0)
        cur["concentrations"] = y
        ys.append(y)
    np.savez_compressed(os.path.join(HERE, "readme_global.npz"), y_solves=np.array(ys), **inp)


if __name__ == "__main__":
    if not oracle.reference_available():
        raise SystemExit("oracle/_ref/libmicm_ref.so is not built (make -C oracle)")
    kernels("syn210", synthetic.synthetic_mechanism(210, 440, seed=2101), 4, 5)
    kernels("syn60", synthetic.synthetic_mechanism(60, 120, seed=601), 6, 6)
    solves("syn60", synthetic.synthetic_mechanism(60, 120, seed=601), 24, 602, 4, 3600.0, {})
    solves("syn210", synthetic.synthetic_mechanism(210, 440, seed=2101), 6, 2103, 4, 600.0,
           dict(t_range=(200.0, 310.0), night_fraction=0.5))
    readme()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
