"""A -k1-> B -k2-> C against its closed form for every rate-constant family of
micm's analytical integration tests (test/integration/analytical_policy.hpp:
TestSimpleSystem :138-276 with TestAnalyticalTroe :409-477, Photolysis
:573-634, TernaryChemicalActivation :723-794, Tunneling :891-950, Arrhenius
:1034-1092, Branched :1177-1263): three cells at micm's temperatures and
pressures, A(0) = 1 - i/3, 999 solves of 1 s, every step compared with the
closed form within micm's absolute tolerance for that family, and the rate
constants within 1e-9 relative.  The C restatement runs every tableau micm
runs these with (2-, 3-, 4-stage, 4- and 6-stage DA); the GPU runs the plain
kernels (one step size for the three cells, as micm) and the fused kernel
(per cell) with the 3-stage tableau."""
import math

import numpy as np
import pytest

import oracle
from micm_b200.mechanism import (GAS_CONSTANT, Mechanism, arrhenius, branched, ternary, troe, tunneling,
                                 user_defined)

TEMPERATURES = [272.5, 254.7, 312.6]
PRESSURES = [101253.3, 100672.5, 101319.8]
NSTEPS = 1000


def _falloff_k(A, B, C, T):
    return A * math.exp(C / T) * math.pow(T / 300.0, B)


def _troe_k1(T, P, rho):
    k0, kinf = 4.0e-11, 1.0
    return k0 * rho / (1.0 + k0 * rho / kinf) * math.pow(0.6, 1.0 / (1.0 + math.pow(math.log10(k0 * rho / kinf), 2)))


def _troe_k2(T, P, rho):
    k0, kinf = _falloff_k(1.2e-3, 1.6, 3.0, T), _falloff_k(136.0, 5.0, 24.0, T)
    return k0 * rho / (1.0 + k0 * rho / kinf) * math.pow(0.9, 0.8 / (0.8 + math.pow(math.log10(k0 * rho / kinf), 2)))


def _ternary_k1(T, P, rho):
    k0, kinf = 4.0e-5, 1.0
    return k0 / (1.0 + k0 * rho / kinf) * math.pow(0.6, 1.0 / (1.0 + math.pow(math.log10(k0 * rho / kinf), 2)))


def _ternary_k2(T, P, rho):
    k0, kinf = _falloff_k(1.2e-3, 1.6, 3.0, T), _falloff_k(136.0, 5.0, 24.0, T)
    return k0 / (1.0 + k0 * rho / kinf) * math.pow(0.9, 0.8 / (0.8 + math.pow(math.log10(k0 * rho / kinf), 2)))


def _branched(T, rho, nitrate):
    a = 2.0e-22 * math.exp(2) * 2.45e19
    b = 0.43 * math.pow(293.0 / 298.0, -8.0)
    z = a / (1.0 + a / b) * math.pow(0.41, 1.0 / (1.0 + math.pow(math.log10(a / b), 2))) * (1.0 - 1.0e-3) / 1.0e-3
    a = 2.0e-22 * math.exp(2) * rho * 6.02214076e23 * 1.0e-6
    b = 0.43 * math.pow(T / 298.0, -8.0)
    A = a / (1.0 + a / b) * math.pow(0.41, 1.0 / (1.0 + math.pow(math.log10(a / b), 2)))
    pre = 1e-4 * math.exp(-204.3 / T)
    return pre * (A / (z + A)) if nitrate else pre * (z / (z + A))


# family -> (rate of A -> B, rate of B -> C, custom parameters per cell, k1(T, P, rho), k2(T, P, rho), tolerance)
FAMILIES = {
    "troe": (troe(k0_A=4.0e-11), troe(1.2e-3, 1.6, 3.0, 136.0, 5.0, 24.0, 0.9, 0.8), [],
             _troe_k1, _troe_k2, 1e-10),
    "photolysis": (user_defined("photoA"), user_defined("photoB"), [2e-3, 3e-3],
                   lambda T, P, rho: 2e-3, lambda T, P, rho: 3e-3, 2e-6),
    "ternary_chemical_activation": (ternary(k0_A=4.0e-5, kinf_A=1.0), ternary(1.2e-3, 1.6, 3.0, 136.0, 5.0, 24.0, 0.9, 0.8),
                                    [], _ternary_k1, _ternary_k2, 1e-8),
    "tunneling": (tunneling(A=4.0e-3), tunneling(A=1.2e-4, B=167.0, C=1.0e8), [],
                  lambda T, P, rho: 4.0e-3,
                  lambda T, P, rho: 1.2e-4 * math.exp(-167 / T + 1.0e8 / math.pow(T, 3)), 1e-8),
    "arrhenius": (arrhenius(A=4.0e-3, C=50.0), arrhenius(A=1.2e-4, B=7.0, C=75.0, D=50.0, E=0.5), [],
                  lambda T, P, rho: 4.0e-3 * math.exp(50 / T),
                  lambda T, P, rho: 1.2e-4 * math.exp(75 / T) * math.pow(T / 50, 7) * (1.0 + 0.5 * P), 1e-9),
    "branched": (branched(0, 1e-4, 204.3, 1.0e-3, 2), branched(1, 1e-4, 204.3, 1.0e-3, 2), [],
                 lambda T, P, rho: _branched(T, rho, False), lambda T, P, rho: _branched(T, rho, True), 1e-13),
}


# micm passes the 2-stage tableau looser tolerances for these families
# (test/integration/test_analytical_rosenbrock.cpp:385, 448, 511)
TWO_STAGE_TOLERANCE = {"tunneling": 2e-5, "arrhenius": 4e-6, "branched": 1e-10}


def tolerance(family, tableau):
    if tableau == 2 and family in TWO_STAGE_TOLERANCE:
        return TWO_STAGE_TOLERANCE[family]
    return FAMILIES[family][5]


def system(family):
    r1, r2 = FAMILIES[family][:2]
    m = Mechanism(species=["A", "B", "C"], reactions=[], name=family)
    m.add(r1, [0], [(1, 1.0)])
    m.add(r2, [1], [(2, 1.0)])
    return m


def inputs(family):
    T, P = np.array(TEMPERATURES), np.array(PRESSURES)
    rho = P / (GAS_CONSTANT * T)
    params = np.tile(np.array(FAMILIES[family][2], dtype=np.float64), (3, 1)).reshape(3, -1)
    y0 = np.array([[1.0 - i / 3.0, 0.0, 0.0] for i in range(3)])
    return dict(temperature=T, pressure=P, air_density=rho, concentrations=y0, custom_params=params)


def closed_form(family, inp, t):
    k1f, k2f = FAMILIES[family][3:5]
    out = np.empty((3, 3))
    for i in range(3):
        T, P, rho = inp["temperature"][i], inp["pressure"][i], inp["air_density"][i]
        k1, k2, a0 = k1f(T, P, rho), k2f(T, P, rho), inp["concentrations"][i, 0]
        out[i, 0] = a0 * math.exp(-k1 * t)
        out[i, 1] = a0 * (k1 / (k2 - k1)) * (math.exp(-k1 * t) - math.exp(-k2 * t))
        out[i, 2] = a0 * (1.0 + (k1 * math.exp(-k2 * t) - k2 * math.exp(-k1 * t)) / (k2 - k1))
    return out


def expected_rates(family, inp):
    k1f, k2f = FAMILIES[family][3:5]
    return np.array([[k1f(T, P, r), k2f(T, P, r)]
                     for T, P, r in zip(inp["temperature"], inp["pressure"], inp["air_density"])])


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("tableau", [2, 3, 4, 40, 60])
@pytest.mark.parametrize("family", sorted(FAMILIES))
def test_restatement_matches_closed_form(family, tableau):
    tol = tolerance(family, tableau)
    R = oracle.Restatement(system(family), tableau_kind=tableau)
    inp = inputs(family)
    k = R.rate_constants(inp["temperature"], inp["pressure"], inp["air_density"], inp["custom_params"])
    # rate constants come in micm's columns; reaction r sits in column reaction_columns[r]
    np.testing.assert_allclose(k[:, R.reaction_columns], expected_rates(family, inp), rtol=1e-9)
    cur = dict(inp)
    for step in range(1, NSTEPS):
        y, stats = R.solve_per_cell(cur, 1.0, threads=1)
        assert np.all(stats[:, 7] == 2)
        cur = dict(cur, concentrations=y)
        np.testing.assert_allclose(y, closed_form(family, inp, float(step)), rtol=0, atol=tol)


@pytest.mark.gpu
@pytest.mark.parametrize("method,step_control", [("plain", "global"), ("fused", "per_cell")])
@pytest.mark.parametrize("family", sorted(FAMILIES))
def test_gpu_matches_closed_form(cuda_device, family, method, step_control):
    from micm_b200 import Solver
    from gpu_helpers import make_state
    tol = FAMILIES[family][5]
    inp = inputs(family)
    solver = Solver(system(family), 3, vector_length=3)
    st = make_state(solver, inp)
    cols = solver.compiled.reaction_columns
    for step in range(1, NSTEPS):
        solver.update_state_parameters(st)
        if step == 1:
            np.testing.assert_allclose(st.rate_constants()[:, cols], expected_rates(family, inp), rtol=1e-9)
        res = solver.solve(1.0, st, method=method, step_control=step_control)
        assert res.converged
        st.sync_outputs_to_host()
        np.testing.assert_allclose(st.concentrations(), closed_form(family, inp, float(step)), rtol=0, atol=tol)


# ---------------------------------------------------------------------------
# The "super stiff but analytical" variants (analytical_policy.hpp
# TestSimpleStiffSystem :278-408 with TestAnalyticalStiffTroe :479-572 and the
# other Stiff* families): A split into A1 and A2 that convert into each other
# at 4e10 and 3.6e10 s-1, both decaying to B with k1; A = A1 + A2 follows the
# same closed form.  Tolerances are micm's, per family and tableau
# (test/integration/test_analytical_rosenbrock.cpp:356-569).
# ---------------------------------------------------------------------------
def _stiff_arrhenius_k2(T, P, rho):
    return 1.2e-4 * math.exp(75 / T) * math.pow(T / 50, 1.6) * (1.0 + 0.5 * P)


# family -> (rate A -> B (for A1 and A2), rate B -> C, custom parameters, k1, k2, {tableau: tolerance})
STIFF_FAMILIES = {
    "troe": (troe(k0_A=4.0e-11), troe(1.2e-3, 1.6, 3.0, 136.0, 5.0, 24.0, 0.9, 0.8), [],
             _troe_k1, _troe_k2, {t: 1e-5 for t in (2, 3, 4, 40, 60)}),
    "photolysis": (None, user_defined("photoB"), [2e-3, 2e-3, 3e-3],
                   lambda T, P, rho: 2e-3, lambda T, P, rho: 3e-3, {t: 2e-5 for t in (2, 3, 4, 40, 60)}),
    "ternary_chemical_activation": (ternary(k0_A=4.0e-5, kinf_A=1.0), ternary(1.2e-3, 1.6, 3.0, 136.0, 5.0, 24.0, 0.9, 0.8),
                                    [], _ternary_k1, _ternary_k2, {t: 2e-3 for t in (2, 3, 4, 40, 60)}),
    "tunneling": (tunneling(A=4.0e-3), tunneling(A=1.2e-4, B=167.0, C=1.0e8), [],
                  lambda T, P, rho: 4.0e-3, lambda T, P, rho: 1.2e-4 * math.exp(-167 / T + 1.0e8 / math.pow(T, 3)),
                  {t: 1e-4 for t in (2, 3, 4, 40, 60)}),
    "arrhenius": (arrhenius(A=4.0e-3, C=50.0), arrhenius(A=1.2e-4, B=1.6, C=75.0, D=50.0, E=0.5), [],
                  lambda T, P, rho: 4.0e-3 * math.exp(50 / T), _stiff_arrhenius_k2,
                  {2: 1e-4, 3: 2e-5, 4: 2e-5, 40: 2e-5, 60: 1e-5}),
    "branched": (branched(0, 1e-4, 204.3, 1.0e-3, 2), branched(1, 1e-4, 204.3, 1.0e-3, 2), [],
                 lambda T, P, rho: _branched(T, rho, False), lambda T, P, rho: _branched(T, rho, True),
                 {t: 2e-3 for t in (2, 3, 4, 40, 60)}),
}


def stiff_system(family):
    r_ab, r_bc = STIFF_FAMILIES[family][:2]
    m = Mechanism(species=["A1", "A2", "B", "C"], reactions=[], name=family + "_stiff")
    if family == "photolysis":
        m.add(user_defined("photoA1B"), [0], [(2, 1.0)])
        m.add(user_defined("photoA2B"), [1], [(2, 1.0)])
    else:
        m.add(r_ab, [0], [(2, 1.0)])
        m.add(r_ab, [1], [(2, 1.0)])
    m.add(r_bc, [2], [(3, 1.0)])
    m.add(arrhenius(A=4.0e10), [0], [(1, 1.0)])
    m.add(arrhenius(A=0.9 * 4.0e10), [1], [(0, 1.0)])
    return m


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("tableau", [2, 3, 4, 40, 60])
@pytest.mark.parametrize("family", sorted(STIFF_FAMILIES))
def test_restatement_matches_stiff_closed_form(family, tableau):
    k1f, k2f, tols = STIFF_FAMILIES[family][3:6]
    R = oracle.Restatement(stiff_system(family), tableau_kind=tableau)
    T, P = np.array(TEMPERATURES), np.array(PRESSURES)
    rho = P / (GAS_CONSTANT * T)
    params = np.tile(np.array(STIFF_FAMILIES[family][2], dtype=np.float64), (3, 1)).reshape(3, -1)
    a0 = np.array([1.0 - i / 3.0 for i in range(3)])
    y0 = np.stack([0.5 * a0, 0.5 * a0, np.zeros(3), np.zeros(3)], axis=1)
    cur = dict(temperature=T, pressure=P, air_density=rho, concentrations=y0, custom_params=params)
    for step in range(1, NSTEPS):
        y, stats = R.solve_per_cell(cur, 1.0, threads=1)
        assert np.all(stats[:, 7] == 2)
        cur = dict(cur, concentrations=y)
        model = np.stack([y[:, 0] + y[:, 1], y[:, 2], y[:, 3]], axis=1)
        want = np.empty((3, 3))
        for i in range(3):
            k1, k2 = k1f(T[i], P[i], rho[i]), k2f(T[i], P[i], rho[i])
            t = float(step)
            want[i] = [a0[i] * math.exp(-k1 * t), a0[i] * (k1 / (k2 - k1)) * (math.exp(-k1 * t) - math.exp(-k2 * t)),
                       a0[i] * (1.0 + (k1 * math.exp(-k2 * t) - k2 * math.exp(-k1 * t)) / (k2 - k1))]
        np.testing.assert_allclose(model, want, rtol=0, atol=tols[tableau])


# ---------------------------------------------------------------------------
# Surface reaction on an aerosol mode (test/integration/analytical_surface_rxn_policy.hpp:
# foo -> bar + 0.4 baz on a lognormal mode, ten steps of 0.1 / k1, relative
# tolerances per tableau from test_analytical_rosenbrock.cpp:574-578).
# ---------------------------------------------------------------------------
SURFACE_TOLERANCE = {2: 1e-2, 3: 1e-5, 4: 1e-6, 40: 1e-5, 60: 1e-7}


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("tableau", [2, 3, 4, 40, 60])
def test_restatement_matches_surface_closed_form(tableau):
    from micm_b200.mechanism import surface
    gmd, gsd, mw, dg, gamma = 1.0e-6, 0.1, 0.04607, 0.95e-5, 2.0e-2
    T, P = 272.5, 101253.3
    radius = gmd / 2.0 * math.exp(5.0 * math.log(gsd) * math.log(gsd) / 2.0)
    number = 6.0 / (math.pi * math.pow(gmd, 3.0) * math.exp(9.0 / 2.0 * math.log(gsd) * math.log(gsd))) * \
        (2.0e-3 / 1000.0 + 3.0e-3 / 1000.0)
    m = Mechanism(species=["foo", "bar", "baz"], reactions=[], name="surface")
    m.add(surface("foo", dg, mw, gamma), [0], [(1, 1.0), (2, 0.4)])
    R = oracle.Restatement(m, tableau_kind=tableau)
    speed = math.sqrt(8.0 * GAS_CONSTANT / (math.pi * mw) * T)
    k1 = 4.0 * number * math.pi * radius * radius / (radius / dg + 4.0 / (speed * gamma))
    inp = dict(temperature=np.array([T]), pressure=np.array([P]), air_density=np.array([P / (GAS_CONSTANT * T)]),
               concentrations=np.array([[1.0, 0.0, 0.0]]), custom_params=np.array([[radius, number]]))
    k = R.rate_constants(inp["temperature"], inp["pressure"], inp["air_density"], inp["custom_params"])
    assert abs(k[0, 0] - k1) <= 1e-8
    dt = 0.1 / k1
    for i in range(1, 11):
        y, stats = R.solve_per_cell(inp, dt, threads=1)
        assert stats[0, 7] == 2
        inp = dict(inp, concentrations=y)
        foo = math.exp(-k1 * i * dt)
        np.testing.assert_allclose(y[0], [foo, 1.0 - foo, 0.4 * (1.0 - foo)], rtol=SURFACE_TOLERANCE[tableau])
