"""The mechanisms and initial states of micm's own benchmark program
(test/benchmark/micm_bench.cpp): TS1 (MOZART-TS1: 209 state species, 547
reactions -- Arrhenius, Troe, user-defined photolysis and surface reactions
with a third body M; test/benchmark/ts1_mechanism.hpp) and Chapman (9
species, 7 reactions; test/benchmark/chapman_mechanism.hpp).  micm_bench
solves them with ThreeStageRosenbrockParameters and dt = 30 s by default.

Each mechanism and its initial state are read from
tests/golden/<name>_mechanism.json, which tests/golden/make_micm_bench.py
writes from micm itself (micm builds the mechanism from the benchmark's code
and the program prints it in this repository's JSON description; see
micm_b200.mechanism.mechanism_from_dict).
"""
from __future__ import annotations

import json
import os
from typing import Dict, Optional

import numpy as np

from .mechanism import Mechanism, ideal_air_density, mechanism_from_dict

GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")
NAMES = ("ts1", "chapman")
TABLEAU = 3          # micm_bench: RosenbrockSolverParameters::ThreeStageRosenbrockParameters()
DT = 30.0            # micm_bench's default time step [s]


def fixture(name: str) -> str:
    if name not in NAMES:
        raise ValueError(f"unknown micm_bench mechanism '{name}' (one of {NAMES})")
    return os.path.join(GOLDEN, f"{name}_mechanism.json")


def document(name: str, path: Optional[str] = None) -> dict:
    with open(path or fixture(name)) as f:
        return json.load(f)


def mechanism(name: str, path: Optional[str] = None, absolute_tolerance: Optional[float] = None) -> Mechanism:
    """The mechanism as micm builds it.  The absolute tolerance is micm's
    builder default (1e-3, what micm_bench runs with) unless one is given for
    every species."""
    m = mechanism_from_dict(document(name, path))
    if absolute_tolerance is not None:
        m.absolute_tolerance = np.full(m.n_species, float(absolute_tolerance))
    return m


def inputs(name: str, n_cells: int, seed: Optional[int] = None, path: Optional[str] = None) -> Dict[str, np.ndarray]:
    """micm_bench's initial state on every cell (its temperature, pressure and
    air density -- Chapman's InitState leaves the air density at 0 --, its
    concentrations and photolysis / aerosol parameters).  With a seed, each
    cell is varied: concentrations scaled by 10**U(-0.5, 0.5), T shifted by
    U(-30, 10) K (air density recomputed) and photolysis rates scaled by
    U(0, 1)."""
    doc = document(name, path)
    mech = mechanism_from_dict(doc)
    init = doc["init"]
    y = np.array([init["concentrations"][s] for s in mech.species], dtype=np.float64)
    labels = mech.custom_param_labels()
    p = np.array([init["custom_parameters"][l] for l in labels], dtype=np.float64)
    n = int(n_cells)
    T = np.full(n, float(init["temperature"]))
    P = np.full(n, float(init["pressure"]))
    rho = np.full(n, float(init["air_density"]))
    conc = np.tile(y, (n, 1))
    params = np.tile(p, (n, 1)).reshape(n, len(labels))
    if seed is not None:
        rng = np.random.default_rng(seed)
        conc *= 10.0 ** rng.uniform(-0.5, 0.5, size=conc.shape)
        T += rng.uniform(-30.0, 10.0, size=n)
        rho = ideal_air_density(P, T)
        photolysis = np.array([l.startswith("j") for l in labels], dtype=bool)
        params[:, photolysis] *= rng.uniform(0.0, 1.0, size=(n, int(photolysis.sum())))
    return dict(temperature=T, pressure=P, air_density=rho, concentrations=conc, custom_params=params)


def micm_columns(name: str, path: Optional[str] = None) -> Dict[str, Dict[str, int]]:
    """micm's own state columns for every species and custom parameter."""
    return document(name, path)["micm_columns"]


def golden(name: str):
    """micm's results on the fixture's 4-cell state (tests/golden/<name>_micm.npz)."""
    return np.load(os.path.join(GOLDEN, f"{name}_micm.npz"))


# ---------------------------------------------------------------------------
# micm_bench's command line (test/benchmark/micm_bench.cpp,
# test/benchmark/bench_harness.hpp), so scripts that drive micm's benchmark
# can drive this library:
#
#   python -m micm_b200.micm_bench [num_cells] [num_steps] [dt_seconds] [backend] [matrix]
#                                  [lu_type] [lu_algorithm] [mechanism]
#
# Same defaults, same "list" and error messages, same result line.  Backends:
# "gpu" is micm's CUDA path (the plain per-stage kernels, one step size for
# all cells); "gpu-fused" is this library's fused kernel with per-cell step
# control.  Matrix "vector1|2|4|8|128" is the state's vector length; the LU
# is the in-place Mozart one.
# ---------------------------------------------------------------------------
VECTOR_WIDTHS = (1, 2, 4, 8, 128)
BACKENDS = {"gpu": ("plain", "global"), "gpu-fused": ("fused", "per_cell")}
USAGE = " [num_cells] [num_steps] [dt_seconds] [backend] [matrix] [lu_type] [lu_algorithm] [mechanism]"


def bench_keys():
    return sorted(f"{m}/{b}/vector{L}/in-place/mozart" for m in NAMES for b in BACKENDS for L in VECTOR_WIDTHS)


def run_case(mechanism_name: str, backend: str, vector_length: int, num_cells: int, num_steps: int,
             dt: float) -> float:
    """bench_harness.hpp RunCase + TimeSolve: build, GetState, the benchmark's
    initial state, UpdateStateParameters once, one converged warm-up Solve,
    num_steps timed Solve(dt) calls on the same state, one converged check
    Solve.  Returns the elapsed milliseconds of the timed calls."""
    import time
    from .solver import Solver
    method, step_control = BACKENDS[backend]
    solver = Solver(mechanism(mechanism_name), TABLEAU, vector_length=vector_length)
    state = solver.get_state(num_cells)
    state.set_inputs(inputs(mechanism_name, num_cells))
    state.sync_inputs_to_device()
    solver.update_state_parameters(state)

    def require_converged(result, when):
        if not result.converged:
            raise RuntimeError(f"the {when} solve did not converge ({result.state}) at dt={dt}; "
                               "reduce dt or correct the initial conditions")

    require_converged(solver.solve(dt, state, method=method, step_control=step_control), "warm-up")
    t0 = time.perf_counter()
    for _ in range(num_steps):
        solver.solve(dt, state, method=method, step_control=step_control)
    elapsed_ms = (time.perf_counter() - t0) * 1e3
    require_converged(solver.solve(dt, state, method=method, step_control=step_control), "post-loop")
    return elapsed_ms


def main(argv=None) -> int:
    import sys
    argv = list(sys.argv if argv is None else argv)
    prog = argv[0] if argv else "micm_bench"
    args = argv[1:]
    if args and args[0] == "list":
        for key in bench_keys():
            print(key)
        return 0
    try:
        num_cells = int(args[0]) if len(args) > 0 else 10000
        num_steps = int(args[1]) if len(args) > 1 else 100
        dt = float(args[2]) if len(args) > 2 else 30.0
        if num_cells < 0 or num_steps < 0:
            raise ValueError("negative count")
    except ValueError as e:
        print(f"Could not read the arguments: {e}")
        print(f"Usage: {prog}{USAGE}")
        return 1
    backend = args[3] if len(args) > 3 else "cpu"
    matrix = args[4] if len(args) > 4 else "standard"
    lu_matrix = args[5] if len(args) > 5 else "in-place"
    lu = args[6] if len(args) > 6 else "mozart"
    mech = args[7] if len(args) > 7 else "chapman"
    key = f"{mech}/{backend}/{matrix}/{lu_matrix}/{lu}"
    if key not in bench_keys():
        print(f"Invalid option combination: {key}")
        print(f"Run '{prog} list' to print every valid combination.")
        return 1
    try:
        elapsed_ms = run_case(mech, backend, int(matrix[len("vector"):]), num_cells, num_steps, dt)
    except Exception as e:  # noqa: BLE001 -- micm_bench reports any failure this way
        print(f"Benchmark failed: {e}")
        return 1
    per_step = elapsed_ms / num_steps if num_steps else float("nan")
    print(f"mechanism={mech} backend={backend} matrix_type={matrix} lu={lu}/{lu_matrix} cells={num_cells} "
          f"steps={num_steps} dt={dt:g} elapsed_ms={elapsed_ms:.3f} ms_per_step={per_step:.3f}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
