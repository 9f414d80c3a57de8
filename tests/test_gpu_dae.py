"""Algebraic constraints (DAE form) on the GPU, per-cell step control (each
cell as micm solves a 1-cell State): the plain per-stage kernels and the
one-cell-per-thread fused kernel against the C restatement of micm's DAE
Rosenbrock in its correctly rounded mode (the GPU's exp/pow are correctly
rounded), bit for bit with identical statistics, and against micm itself within
rtol 1e-6 with identical accepted-step counts.  micm's CUDA path rejects
constraints (solver_builder.inl:251-266); its CPU path is the reference."""
import numpy as np
import pytest

import oracle
from micm_b200 import Solver

from gpu_helpers import make_state
from test_dae import CASES

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (oracle.restatement_available() and oracle.reference_available()),
                                 reason="oracle not built")]
STATS = ("function_calls", "jacobian_updates", "number_of_steps", "accepted", "rejected", "decompositions", "solves")


@pytest.mark.parametrize("method", ["plain", "fused"])
@pytest.mark.parametrize("name,make_mech,make_inputs,tableau,outputs", CASES, ids=[c[0] for c in CASES])
def test_gpu_equals_correctly_rounded_restatement(cuda_device, method, name, make_mech, make_inputs, tableau,
                                                  outputs):
    m = make_mech()
    inp = make_inputs(m)
    R = oracle.Restatement(m, tableau_kind=tableau, correctly_rounded=True)
    solver = Solver(m, tableau, vector_length=4)
    st = make_state(solver, inp)
    solver.update_state_parameters(st)
    y_r = inp["concentrations"]
    t = 0.0
    for target in outputs:
        dt = target - t
        y_r, st_r = R.solve_per_cell(dict(inp, concentrations=y_r), dt, threads=1)
        res = solver.solve(dt, st, method=method, step_control="per_cell", per_cell=True)
        st.sync_outputs_to_host()
        np.testing.assert_array_equal(st.concentrations(), y_r)
        np.testing.assert_array_equal(res.per_cell_status, st_r[:, 7])
        np.testing.assert_array_equal(res.per_cell_accepted, st_r[:, 3])
        for q, key in enumerate(STATS):
            assert res.stats[key] == st_r[:, q].sum(), key
        assert res.stats["constraint_init_iterations"] == st_r[:, 9].sum()
        t = target


CONVERGING = [c for c in CASES if c[0] != "equilibrium_singular_init"]


@pytest.mark.parametrize("name,make_mech,make_inputs,tableau,outputs", CASES, ids=[c[0] for c in CASES])
def test_gpu_global_equals_correctly_rounded_restatement(cuda_device, name, make_mech, make_inputs, tableau,
                                                         outputs):
    """micm's n-cell State (one step size for every cell): the constraint
    initialisation's residual maximum over all cells decides on the device."""
    m = make_mech()
    inp = make_inputs(m)
    R = oracle.Restatement(m, tableau_kind=tableau, correctly_rounded=True)
    solver = Solver(m, tableau, vector_length=32)
    st = make_state(solver, inp)
    solver.update_state_parameters(st)
    y_r = inp["concentrations"]
    t = 0.0
    for target in outputs:
        dt = target - t
        y_r, st_r = R.solve_global(dict(inp, concentrations=y_r), dt)
        res = solver.solve(dt, st, method="plain", step_control="global")
        st.sync_outputs_to_host()
        np.testing.assert_array_equal(st.concentrations(), y_r)
        assert res.state == st_r[7]
        for q, key in enumerate(STATS):
            assert res.stats[key] == st_r[q], key
        assert res.stats["constraint_init_iterations"] == st_r[9]
        t = target


@pytest.mark.parametrize("name,make_mech,make_inputs,tableau,outputs", CONVERGING, ids=[c[0] for c in CONVERGING])
def test_gpu_follows_micm(cuda_device, name, make_mech, make_inputs, tableau, outputs):
    m = make_mech()
    inp = make_inputs(m)
    ref = oracle.Reference(m, tableau=tableau)
    solver = Solver(m, tableau, vector_length=4)
    st = make_state(solver, inp)
    solver.update_state_parameters(st)
    y_m = inp["concentrations"]
    t = 0.0
    same = total = 0
    for target in outputs:
        dt = target - t
        y_m, st_m = ref.solve_per_cell(dict(inp, concentrations=y_m), dt, threads=1)
        res = solver.solve(dt, st, method="fused", step_control="per_cell", per_cell=True)
        st.sync_outputs_to_host()
        np.testing.assert_allclose(st.concentrations(), y_m, rtol=1e-6, atol=1e-12)
        same += int(np.sum(res.per_cell_accepted == st_m[:, 3]))
        total += len(st_m)
        t = target
    assert same >= 0.9 * total


@pytest.mark.parametrize("method,step_control", [("plain", "global"), ("plain", "per_cell"), ("fused", "per_cell")])
def test_gpu_micm_constraint_initialisation_cases(cuda_device, method, step_control):
    """micm's ConstraintInitialization unit tests on the GPU: the three-cell
    State (consistent, mildly and severely inconsistent cells), then C
    perturbed to 999 in every cell and solved again; equal to the correctly
    rounded restatement bit for bit, with the tests' expectations."""
    from dae_cases import SIMPLE_MULTICELL, simple_constrained, simple_inputs
    m = simple_constrained()
    inp = simple_inputs(SIMPLE_MULTICELL)
    R = oracle.Restatement(m, tableau_kind=3, correctly_rounded=True)
    solver = Solver(m, 3, vector_length=4)
    st = make_state(solver, inp)
    solver.update_state_parameters(st)
    y = inp["concentrations"]
    for round_ in range(2):
        if step_control == "global":
            y, st_r = R.solve_global(dict(inp, concentrations=y), 0.001)
            iters = st_r[9]
        else:
            y, st_r = R.solve_per_cell(dict(inp, concentrations=y), 0.001, threads=1)
            iters = st_r[:, 9].sum()
        res = solver.solve(0.001, st, method=method, step_control=step_control)
        st.sync_outputs_to_host()
        np.testing.assert_array_equal(st.concentrations(), y)
        assert res.state == 2 and res.stats["constraint_init_iterations"] == iters
        assert np.all(np.abs(2.0 * y[:, 1] - y[:, 2]) < 1e-5)
        y = y.copy()
        y[:, 2] = 999.0
        st.set_concentrations(y)
        st.sync_inputs_to_device()
