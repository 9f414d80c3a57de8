"""The FP64 discrete-adjoint oracle against central finite differences.

The adjoint differentiates the accepted Rosenbrock steps with their step
sizes held fixed, so the finite differences are taken of that map: the
oracle's fixed-step replay of the accepted step sizes (which reproduces the
adaptive solve bit for bit).  Entries are compared where the output is
sensitive to them (at least 1e-3 of the largest sensitivity of that cell);
the others are below the roundoff of a difference quotient.
"""
import numpy as np
import pytest

import oracle
from micm_b200 import synthetic

pytestmark = pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")


@pytest.fixture(scope="module")
def case():
    cfg = synthetic.CONFIGS["c60_adjoint"]
    mech = cfg["mech"]()
    inputs = synthetic.cell_inputs(mech, 3, 7, **cfg["inputs"])
    R = oracle.Restatement(mech, tableau_kind=cfg["stages"])
    k = R._k(inputs)
    h, steps = R.step_sizes_per_cell(inputs, cfg["dt"], 512, k)
    return cfg, mech, inputs, R, k, h, steps


def test_replay_reproduces_solve(case):
    cfg, mech, inputs, R, k, h, steps = case
    y_solve, _ = R.solve_per_cell(inputs, cfg["dt"], k=k)
    y_replay = R.replay_per_cell(inputs["concentrations"], k, h, steps)
    np.testing.assert_array_equal(y_solve, y_replay)
    assert steps.min() > 10


@pytest.mark.parametrize("species", [0, 5])
def test_adjoint_matches_finite_differences(case, species):
    cfg, mech, inputs, R, k, h, steps = case
    y0 = inputs["concentrations"]
    y_final, _ = R.solve_per_cell(inputs, cfg["dt"], k=k)
    ybar = np.zeros_like(y_final)
    ybar[:, species] = 1.0
    _, g0, gk = R.adjoint_per_cell(inputs, cfg["dt"], ybar, k=k)

    def out(y, kk=k):
        return R.replay_per_cell(y, kk, h, steps)[:, species]

    rel_h = 1e-6  # relative perturbation of the finite differences
    worst = 0.0
    imp = np.abs(g0) * np.abs(y0)
    for j in range(mech.n_species):
        e = rel_h * np.abs(y0[:, j])
        yp, ym = y0.copy(), y0.copy()
        yp[:, j] += e
        ym[:, j] -= e
        fd = (out(yp) - out(ym)) / (2 * e)
        sig = imp[:, j] > 1e-3 * imp.max(axis=1)
        if sig.any():
            worst = max(worst, (np.abs(fd - g0[:, j]) / np.abs(g0[:, j]))[sig].max())
    kimp = np.abs(gk)
    for r in range(mech.n_reactions):
        c = R.reaction_columns[r]
        kp, km = k.copy(), k.copy()
        kp[:, c] *= np.exp(rel_h)
        km[:, c] *= np.exp(-rel_h)
        fd = (out(y0, kp) - out(y0, km)) / (2 * rel_h)
        sig = kimp[:, r] > 1e-3 * kimp.max(axis=1)
        if sig.any():
            worst = max(worst, (np.abs(fd - gk[:, r]) / np.abs(gk[:, r]))[sig].max())
    assert worst < 1e-5


def test_adjoint_on_micms_ts1_mechanism_matches_finite_differences():
    """The same check on micm's TS1 benchmark mechanism (Troe, photolysis,
    surface reactions, a third body), two varied cells, gradients of the final
    O3 (absolute tolerance 1e-9, 3-stage Rosenbrock, dt = 30 s)."""
    from micm_b200 import ts1
    mech = ts1.mechanism(absolute_tolerance=1e-9)
    inputs = ts1.inputs(2, seed=5)
    R = oracle.Restatement(mech, tableau_kind=ts1.TABLEAU)
    k = R._k(inputs)
    h, steps = R.step_sizes_per_cell(inputs, ts1.DT, 1024, k)
    y_final, _ = R.solve_per_cell(inputs, ts1.DT, k=k)
    np.testing.assert_array_equal(R.replay_per_cell(inputs["concentrations"], k, h, steps), y_final)
    o3 = mech.species.index("O3")
    ybar = np.zeros_like(y_final)
    ybar[:, o3] = 1.0
    _, g0, gk = R.adjoint_per_cell(inputs, ts1.DT, ybar, k=k, max_steps=1024)

    def out(y, kk=k):
        return R.replay_per_cell(y, kk, h, steps)[:, o3]

    rel_h, worst, checked = 1e-6, 0.0, 0
    y0 = inputs["concentrations"]
    imp = np.abs(g0) * np.abs(y0)
    for j in range(mech.n_species):
        e = rel_h * np.abs(y0[:, j])
        sig = imp[:, j] > 1e-3 * imp.max(axis=1)
        if not sig.any() or np.any(e[sig] == 0):
            continue
        yp, ym = y0.copy(), y0.copy()
        yp[:, j] += e
        ym[:, j] -= e
        fd = (out(yp) - out(ym)) / (2 * np.where(e > 0, e, 1.0))
        worst = max(worst, (np.abs(fd - g0[:, j]) / np.abs(g0[:, j]))[sig].max())
        checked += 1
    kimp = np.abs(gk)
    for r in range(mech.n_reactions):
        sig = kimp[:, r] > 1e-3 * kimp.max(axis=1)
        if not sig.any():
            continue
        c = R.reaction_columns[r]
        kp, km = k.copy(), k.copy()
        kp[:, c] *= np.exp(rel_h)
        km[:, c] *= np.exp(-rel_h)
        fd = (out(y0, kp) - out(y0, km)) / (2 * rel_h)
        worst = max(worst, (np.abs(fd - gk[:, r]) / np.abs(gk[:, r]))[sig].max())
        checked += 1
    assert checked > 10 and worst < 1e-5
