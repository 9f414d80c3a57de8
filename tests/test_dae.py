"""Algebraic constraints (DAE form): micm's Rosenbrock with linear and
equilibrium constraints (include/micm/constraint/**, rosenbrock.inl:12-304 and
InitializeConstraints :407-576), restated in the C oracle and pinned bit for
bit against micm itself (oracle/_ref, micm's constraint classes through
SolverBuilder::SetConstraints), on problems shaped after micm's
test/integration/test_linear_constraint.cpp and test_equilibrium_constraint.cpp:
every solve's final concentrations and statistics (constraint-initialisation
iterations included) are identical."""
import numpy as np
import pytest

import oracle
from dae_cases import (SIMPLE_CONSISTENT, SIMPLE_MILD, SIMPLE_MULTICELL, SIMPLE_SEVERE, equilibrium,
                       equilibrium_inputs, negative_algebraic, negative_algebraic_inputs, simple_constrained,
                       simple_inputs, terminator_robertson, terminator_robertson_inputs)

pytestmark = pytest.mark.skipif(not (oracle.restatement_available() and oracle.reference_available()),
                                reason="oracle not built")

CASES = [
    ("linear_4da", terminator_robertson, lambda m: terminator_robertson_inputs(3), 40, [1, 10, 100, 1e3, 1e4, 1e5]),
    ("linear_6da", terminator_robertson, lambda m: terminator_robertson_inputs(2), 60, [1, 10, 100, 1e3]),
    ("equilibrium_consistent", lambda: equilibrium(), lambda m: equilibrium_inputs(m, 4, True), 40, [1, 5, 20, 60]),
    ("equilibrium_inconsistent_3stage", lambda: equilibrium(), lambda m: equilibrium_inputs(m, 4, False), 3,
     [1, 5, 20]),
    ("equilibrium_stoich2_two", lambda: equilibrium(2.0, True), lambda m: equilibrium_inputs(m, 3, False, 0.2), 40,
     [1, 10, 50]),
    ("negative_algebraic", negative_algebraic, lambda m: negative_algebraic_inputs(3), 40, [1, 10, 30]),
    # F = 0 with F^2 as the product: dG/dF = 0, the initialisation's matrix is
    # singular and micm reports InfDetected
    ("equilibrium_singular_init", lambda: equilibrium(2.0, True), lambda m: equilibrium_inputs(m, 3, False, 0.0), 40,
     [1]),
]


@pytest.mark.parametrize("name,make_mech,make_inputs,tableau,outputs", CASES, ids=[c[0] for c in CASES])
def test_restatement_equals_micm(name, make_mech, make_inputs, tableau, outputs):
    m = make_mech()
    inp = make_inputs(m)
    R = oracle.Restatement(m, tableau_kind=tableau)
    ref = oracle.Reference(m, tableau=tableau)
    y_r, y_m = inp["concentrations"], inp["concentrations"]
    t = 0.0
    for target in outputs:
        dt = target - t
        y_r, st_r = R.solve_per_cell(dict(inp, concentrations=y_r), dt, threads=1)
        y_m, st_m = ref.solve_per_cell(dict(inp, concentrations=y_m), dt, threads=1)
        np.testing.assert_array_equal(y_r, y_m)
        np.testing.assert_array_equal(st_r, st_m)
        assert np.all(st_r[:, 7] == (7 if name == "equilibrium_singular_init" else 2)), st_r[:, 7]
        t = target
    if name.startswith("linear"):
        np.testing.assert_allclose(y_r[:, 2] + y_r[:, 3] + y_r[:, 4], 1.0, rtol=0, atol=1e-10)
    if "inconsistent" in name or "two" in name:
        assert st_r[:, 9].max() >= 1  # the initialisation iterated


@pytest.mark.parametrize("make_mech", [terminator_robertson, lambda: equilibrium(), lambda: equilibrium(2.0, True)],
                         ids=["linear", "equilibrium", "two_equilibria"])
def test_library_numbering_and_pattern_equal_micms(make_mech):
    """The library's compile of a DAE mechanism: micm's species numbering, and
    micm's Jacobian pattern with the algebraic rows' kinetic entries replaced
    by the constraints' (solver_builder.inl:345-393), LU fill included."""
    from micm_b200.solver import CompiledMechanism
    m = make_mech()
    cm = CompiledMechanism(m)
    ref = oracle.Reference(m, tableau=40)
    R = oracle.Restatement(m, tableau_kind=40)
    np.testing.assert_array_equal(cm.species_columns, ref.species_columns)
    np.testing.assert_array_equal(cm.rows, ref.rows)
    np.testing.assert_array_equal(cm.cols, ref.cols)
    np.testing.assert_array_equal(cm.rows, R.rows)
    np.testing.assert_array_equal(cm.cols, R.cols)
    assert cm.info["n_custom_params"] == ref.n_params


def test_invalid_constraints_rejected():
    from micm_b200._native import MicmbError
    from micm_b200.mechanism import linear_constraint
    from micm_b200.solver import CompiledMechanism
    m = terminator_robertson()
    m.constraints.append(linear_constraint(4, [(2, 1.0)], 0.5))  # C is already algebraic
    with pytest.raises(MicmbError):
        CompiledMechanism(m)
    m = terminator_robertson()
    m.constraints[0].terms.append((9, 1.0))  # no such species
    with pytest.raises(MicmbError):
        CompiledMechanism(m)


@pytest.mark.parametrize("name,make_mech,make_inputs,tableau,outputs", CASES, ids=[c[0] for c in CASES])
def test_global_restatement_follows_micms_multicell_state(name, make_mech, make_inputs, tableau, outputs):
    """One n-cell State (micm's global step size): the constraint
    initialisation iterates all cells until the largest residual of any cell
    meets the tolerance, then one step size serves every cell.  The
    restatement sums the error norm in the GPU's fixed order and micm with one
    accumulator, so values agree to rounding and the counts exactly."""
    m = make_mech()
    inp = make_inputs(m)
    R = oracle.Restatement(m, tableau_kind=tableau)
    ref = oracle.Reference(m, tableau=tableau)
    y_r, y_m = inp["concentrations"], inp["concentrations"]
    t = 0.0
    for target in outputs:
        dt = target - t
        y_r, st_r = R.solve_global(dict(inp, concentrations=y_r), dt)
        y_m, st_m = ref.solve_global(dict(inp, concentrations=y_m), dt)
        for q, key in enumerate(oracle.STATS_FIELDS):
            assert st_r[q] == st_m[0][key], key
        assert st_r[9] == st_m[0]["constraint_init_iterations"]
        np.testing.assert_allclose(y_r, y_m, rtol=1e-9, atol=1e-300)
        t = target
    if name == "negative_algebraic":
        assert np.all(y_r[:, 2] < 0.0)  # algebraic variables are not clamped



def _residual(y):
    return 2.0 * y[:, 1] - y[:, 2]


@pytest.mark.parametrize("rows,max_iters,min_iters", [([SIMPLE_CONSISTENT], 1, 0), ([SIMPLE_MILD], 10, 1),
                                                      ([SIMPLE_SEVERE], 10, 1)],
                         ids=["consistent", "mildly_inconsistent", "severely_inconsistent"])
def test_micm_constraint_initialisation_cases(rows, max_iters, min_iters):
    """micm's ConstraintInitialization unit tests (3-stage tableau, one 1-cell
    State, Solve(0.001)): the restatement equals micm bit for bit and both
    meet the tests' expectations (converged, residual below 1e-6,
    initialisation iterations as the tests bound them)."""
    m = simple_constrained()
    inp = simple_inputs(rows)
    y_r, st_r = oracle.Restatement(m, tableau_kind=3).solve_per_cell(inp, 0.001, threads=1)
    y_m, st_m = oracle.Reference(m, tableau=3).solve_per_cell(inp, 0.001, threads=1)
    np.testing.assert_array_equal(y_r, y_m)
    np.testing.assert_array_equal(st_r, st_m)
    assert st_r[0, 7] == 2
    assert min_iters <= st_r[0, 9] <= max_iters
    assert abs(_residual(y_r)[0]) < 1e-6


def test_micm_multicell_initialisation_and_reinitialisation():
    """micm's MultiCellSystems test (one 3-cell State: consistent, mildly and
    severely inconsistent cells) and SubsequentSolveCallsReinitialize (C
    perturbed to 999 between solves), restatement against micm."""
    m = simple_constrained()
    inp = simple_inputs(SIMPLE_MULTICELL)
    R = oracle.Restatement(m, tableau_kind=3)
    ref = oracle.Reference(m, tableau=3)
    y_r, st_r = R.solve_global(inp, 0.001)
    y_m, st_m = ref.solve_global(inp, 0.001)
    np.testing.assert_allclose(y_r, y_m, rtol=1e-12, atol=0)
    for q, key in enumerate(oracle.STATS_FIELDS):
        assert st_r[q] == st_m[0][key], key
    assert st_r[7] == 2 and st_r[9] == st_m[0]["constraint_init_iterations"] >= 2
    assert np.all(np.abs(_residual(y_r)) < 1e-5)
    one = simple_inputs([SIMPLE_CONSISTENT])
    y1, s1 = R.solve_per_cell(one, 0.001, threads=1)
    y1[0, 2] = 999.0
    y2, s2 = R.solve_per_cell(dict(one, concentrations=y1), 0.001, threads=1)
    y2m, s2m = ref.solve_per_cell(dict(one, concentrations=y1), 0.001, threads=1)
    np.testing.assert_array_equal(y2, y2m)
    np.testing.assert_array_equal(s2, s2m)
    assert s1[0, 7] == 2 and s2[0, 7] == 2 and s2[0, 9] >= 2
    assert abs(_residual(y2)[0]) < 1e-6


def _advance_both(m, inp, tableau, dt):
    """micm's loop (Solve(dt - advanced) until the interval is covered) run by
    the restatement and by micm; every call equal bit for bit.  Returns the
    states after each call."""
    R = oracle.Restatement(m, tableau_kind=tableau)
    ref = oracle.Reference(m, tableau=tableau)
    y, advanced, states = inp["concentrations"], 0.0, []
    while advanced < dt:
        y_r, st_r = R.solve_per_cell(dict(inp, concentrations=y), dt - advanced, threads=1)
        y_m, st_m = ref.solve_per_cell(dict(inp, concentrations=y), dt - advanced, threads=1)
        np.testing.assert_array_equal(y_r, y_m)
        np.testing.assert_array_equal(st_r, st_m)
        assert st_r[0, 7] == 2
        advanced += float(st_r[0:1, 8:9].view(np.float64)[0, 0])
        y = y_r
        states.append(y[0].copy())
    return states


@pytest.mark.parametrize("tableau", [40, 3, 4, 60], ids=["4da", "3", "4", "6da"])
def test_micm_overshoot_linear(tableau):
    """micm's AlgebraicVariableStaysNonNegative (4-stage DA) and
    AllRosenbrockOrdersConstrained (2-stage excluded as micm does): 30 s of a
    fast A -> B under A + B + C = 1e-6; the restatement equals micm on every
    Solve call, and micm's assertions hold."""
    from dae_cases import overshoot_linear, overshoot_linear_inputs
    states = _advance_both(overshoot_linear(), overshoot_linear_inputs(), tableau, 30.0)
    for s in states:
        assert abs(s.sum() - 1.0e-6) < 1e-12
        assert s[2] >= -1.0e-18
    a, b, c = states[-1]
    assert a < 1e-12 and abs(b - 0.9e-6) < 1e-10 and abs(c - 0.1e-6) < 1e-10


def test_micm_overshoot_equilibrium_plus_conservation():
    """micm's EquilibriumPlusConservation: an equilibrium and a linear
    constraint together (two algebraic rows), restatement equal to micm."""
    from dae_cases import overshoot_equilibrium, overshoot_equilibrium_inputs
    states = _advance_both(overshoot_equilibrium(), overshoot_equilibrium_inputs(), 40, 30.0)
    for s in states:
        assert abs(s.sum() - 1.0e-6) < 1e-12
        assert s[0] >= -1.0e-8


def _accepted(m, inp, dt):
    """restatement == micm on every call of micm's loop; (states, accepted steps)"""
    R = oracle.Restatement(m, tableau_kind=40)
    ref = oracle.Reference(m, tableau=40)
    y, advanced, states, acc = inp["concentrations"], 0.0, [], 0
    while advanced < dt:
        y_r, st_r = R.solve_per_cell(dict(inp, concentrations=y), dt - advanced, threads=1)
        y_m, st_m = ref.solve_per_cell(dict(inp, concentrations=y), dt - advanced, threads=1)
        np.testing.assert_array_equal(y_r, y_m)
        np.testing.assert_array_equal(st_r, st_m)
        assert st_r[0, 7] == 2
        advanced += float(st_r[0:1, 8:9].view(np.float64)[0, 0])
        acc += int(st_r[0, 3])
        y = y_r
        states.append(y[0].copy())
    return states, acc


def test_micm_algebraic_error_cascade():
    """micm's DAEAlgebraicError tests: a tight absolute tolerance on the
    balance variable takes more steps than a loose one (the algebraic rows'
    step-change error counts), and the ultra-stiff cascade does not overshoot;
    the restatement equals micm on every call of each run."""
    from dae_cases import cascade
    _, loose = _accepted(*cascade(1e-3, 100.0, 2.0, 2.0), 30.0)
    _, tight = _accepted(*cascade(1e-8, 100.0, 2.0, 2.0), 30.0)
    assert tight > loose
    states, _ = _accepted(*cascade(1e-8, 1.0e4, 100.0, 50.0), 30.0)
    assert min(s[0] for s in states) >= -1.0e-8
    assert abs(states[-1][3] - 1.0e-6) < 1e-8 and abs(states[-1][0]) < 1e-10


@pytest.mark.parametrize("make_mech", [terminator_robertson, lambda: equilibrium(2.0, True)], ids=["linear", "two_eq"])
def test_constraints_round_trip_through_json(make_mech, tmp_path):
    """The JSON mechanism description carries the constraints: written and read
    back, the mechanism compiles to the same numbering and pattern and solves
    the same (restatement) bit for bit."""
    from micm_b200.mechanism import load_mechanism_json, save_mechanism_json
    from micm_b200.solver import CompiledMechanism
    m = make_mech()
    path = str(tmp_path / "mech.json")
    save_mechanism_json(m, path)
    m2 = load_mechanism_json(path)
    assert [(c.kind, c.species, c.terms, c.n_reactants, tuple(c.params)) for c in m2.constraints] == \
        [(c.kind, c.species, c.terms, c.n_reactants, tuple(c.params)) for c in m.constraints]
    a, b = CompiledMechanism(m), CompiledMechanism(m2)
    np.testing.assert_array_equal(a.rows, b.rows)
    np.testing.assert_array_equal(a.cols, b.cols)
    inp = terminator_robertson_inputs(2) if m.n_species == 5 else equilibrium_inputs(m, 2, False, 0.2)
    y1, s1 = oracle.Restatement(m, tableau_kind=40).solve_per_cell(inp, 10.0, threads=1)
    y2, s2 = oracle.Restatement(m2, tableau_kind=40).solve_per_cell(inp, 10.0, threads=1)
    np.testing.assert_array_equal(y1, y2)
    np.testing.assert_array_equal(s1, s2)
