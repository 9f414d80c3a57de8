"""DAE test problems shaped after micm's constraint integration tests
(test/integration/test_linear_constraint.cpp,
test/integration/test_equilibrium_constraint.cpp): mechanisms, inputs and the
driver that advances one state over a sequence of output times the way those
tests do (Solve(time_step - advanced) until the output time is reached)."""
import numpy as np

from micm_b200.mechanism import (Mechanism, arrhenius, equilibrium_constraint, ideal_air_density, linear_constraint,
                                 user_defined)


def terminator_robertson():
    """Cl2 -> 2 Cl, Cl + Cl -> Cl2 and Robertson's A, B, C with the linear
    constraint A + B + C = 1 replacing C's row."""
    atol = np.array([1e-20, 1e-20, 1e-3, 1e-3, 1e-3])
    m = Mechanism(species=["Cl2", "Cl", "A", "B", "C"], reactions=[], name="terminator_robertson",
                  reorder_state=False, absolute_tolerance=atol, relative_tolerance=1e-8)
    m.add(user_defined("terminator_k1"), [0], [(1, 2.0)])
    m.add(arrhenius(A=1.0), [1, 1], [(0, 1.0)])
    m.add(user_defined("robertson_r1"), [2], [(3, 1.0)])
    m.add(user_defined("robertson_r2"), [3, 3], [(3, 1.0), (4, 1.0)])
    m.add(user_defined("robertson_r3"), [3, 4], [(2, 1.0), (4, 1.0)])
    m.constraints.append(linear_constraint(4, [(2, 1.0), (3, 1.0), (4, 1.0)], 1.0, name="mass_conservation"))
    return m


def terminator_robertson_inputs(n=1):
    T = np.full(n, 298.0)
    P = np.full(n, 101300.0)
    y = np.tile([1.8e-10, 1.2e-6, 1.0, 0.0, 0.0], (n, 1))
    y[:, 1] *= np.linspace(1.0, 2.0, n)
    # custom parameters in micm's order: terminator_k1, robertson_r1, r2, r3
    params = np.tile([1.0e-4, 0.04, 3.0e7, 1.0e4], (n, 1))
    return dict(temperature=T, pressure=P, air_density=np.full(n, 42.0), concentrations=y, custom_params=params)


def negative_algebraic():
    """A -> B (k = 0.1) with the linear constraint A + B + C = 1 replacing C's
    row; started from A + B = 1.5 the initialisation sets C to -0.5, which
    micm's post-solve clamp leaves as solved (only ODE variables are clamped)."""
    m = Mechanism(species=["A", "B", "C"], reactions=[], name="negative_algebraic", reorder_state=False,
                  absolute_tolerance=np.full(3, 1e-6), relative_tolerance=1e-6)
    m.add(arrhenius(A=0.1), [0], [(1, 1.0)])
    m.constraints.append(linear_constraint(2, [(0, 1.0), (1, 1.0), (2, 1.0)], 1.0, name="total"))
    return m


def negative_algebraic_inputs(n=3):
    T = np.full(n, 298.0)
    P = np.full(n, 101325.0)
    y = np.tile([1.0, 0.5, 0.0], (n, 1))
    y[:, 0] *= np.linspace(1.0, 1.5, n)
    return dict(temperature=T, pressure=P, air_density=ideal_air_density(P, T), concentrations=y,
                custom_params=np.zeros((n, 0)))


def equilibrium(stoich=1.0, two=False):
    """A -> B (k = 0.1) with B <=> C in equilibrium (C algebraic); with
    `two`, also D -> E with E <=> F.  `stoich` is B's exponent."""
    names = ["A", "B", "C"] + (["D", "E", "F"] if two else [])
    m = Mechanism(species=names, reactions=[], name="equilibrium", reorder_state=False,
                  absolute_tolerance=np.full(len(names), 1e-3), relative_tolerance=1e-6)
    m.add(arrhenius(A=0.1), [0], [(1, 1.0)])
    m.constraints.append(equilibrium_constraint(2, [(1, stoich)], [(2, 1.0)], K_HLC_ref=0.034, delta_H=-2400.0,
                                                name="B_C_eq"))
    if two:
        m.add(arrhenius(A=0.02, C=-300.0), [3], [(4, 1.0)])
        m.constraints.append(equilibrium_constraint(5, [(4, 1.0)], [(5, 2.0)], K_HLC_ref=1.7, delta_H=1800.0,
                                                    name="E_F_eq"))
    return m


def equilibrium_inputs(m, n=4, consistent=True, f0=0.0):
    T = np.linspace(280.0, 310.0, n)
    P = np.full(n, 101325.0)
    S = m.n_species
    y = np.zeros((n, S))
    y[:, 0] = 1.0
    y[:, 1] = 0.1
    if S > 3:
        y[:, 3] = 0.5
        y[:, 4] = 0.05
        y[:, 5] = f0
    if consistent:
        keq = 0.034 * np.exp((-2400.0 / (1.380649e-23 * 6.02214076e23)) * (1.0 / T - 1.0 / 298.15))
        y[:, 2] = keq * y[:, 1] ** m.constraints[0].terms[0][1]
    return dict(temperature=T, pressure=P, air_density=ideal_air_density(P, T), concentrations=y,
                custom_params=np.zeros((n, 0)))


def advance(solve, inputs, output_times):
    """Advance every cell to each output time by repeated solves of the rest of
    the interval; yields (y, per-call stats) per output time.  `solve(inputs,
    dt)` returns (y [n, S], stats rows [n, 10])."""
    t = 0.0
    for target in output_times:
        advanced = 0.0
        calls = []
        while advanced < target - t:
            y, st = solve(inputs, (target - t) - advanced)
            calls.append(st)
            inputs = dict(inputs, concentrations=y)
            ft = st[:, 8:9].view(np.float64)[:, 0]
            if not np.all(ft == ft[0]) or ft[0] <= 0.0:
                raise AssertionError("cells advanced unevenly or not at all")
            advanced += ft[0]
        t = target
        yield inputs["concentrations"], calls


def simple_constrained():
    """micm's constraint-initialisation unit-test system
    (test/unit/solver/test_constraint_initialization.cpp:21-58): A -> B with
    k = 0.5 and the equilibrium constraint C = K_eq B, K_eq = 2 with no
    temperature dependence; micm's builder defaults (absolute tolerance 1e-3,
    relative 1e-6), the species in system order."""
    m = Mechanism(species=["A", "B", "C"], reactions=[], name="simple_constrained", reorder_state=False,
                  absolute_tolerance=np.full(3, 1e-3), relative_tolerance=1e-6)
    m.add(arrhenius(A=0.5), [0], [(1, 1.0)])
    m.constraints.append(equilibrium_constraint(2, [(1, 1.0)], [(2, 1.0)], K_HLC_ref=2.0, delta_H=0.0,
                                                name="B_C_eq"))
    return m


# the unit tests' initial states (A, B, C): consistent, mildly and severely
# inconsistent (test_constraint_initialization.cpp:80-82, :117-119, :163-165),
# and the multi-cell test's three cells (:246-259)
SIMPLE_CONSISTENT = [1.0, 0.5, 1.0]
SIMPLE_MILD = [1.0, 0.5, 5.0]
SIMPLE_SEVERE = [1.0, 0.5, 1000.0]
SIMPLE_MULTICELL = [[1.0, 0.5, 1.0], [2.0, 0.3, 5.0], [0.5, 0.1, 100.0]]


def simple_inputs(rows):
    y = np.array(rows, dtype=float).reshape(-1, 3)
    n = len(y)
    T = np.full(n, 298.15)
    P = np.full(n, 101325.0)
    return dict(temperature=T, pressure=P, air_density=ideal_air_density(P, T), concentrations=y,
                custom_params=np.zeros((n, 0)))


def overshoot_linear():
    """micm's DAE overshoot case (test/integration/test_dae_constraint_overshoot.cpp:44-129):
    a fast A -> B (k = 1e4) with the conservation A + B + C = 1e-6 replacing
    C's row; absolute tolerance 1e-12, relative 1e-6."""
    m = Mechanism(species=["A", "B", "C"], reactions=[], name="overshoot_linear", reorder_state=False,
                  absolute_tolerance=np.full(3, 1e-12), relative_tolerance=1e-6)
    m.add(arrhenius(A=1.0e4), [0], [(1, 1.0)])
    m.constraints.append(linear_constraint(2, [(0, 1.0), (1, 1.0), (2, 1.0)], 1.0e-6, name="mass_conservation"))
    return m


def overshoot_linear_inputs():
    return dict(temperature=np.array([298.0]), pressure=np.array([101325.0]),
                air_density=ideal_air_density(np.array([101325.0]), np.array([298.0])),
                concentrations=np.array([[0.9e-6, 0.0, 0.1e-6]]), custom_params=np.zeros((1, 0)))


def overshoot_equilibrium():
    """micm's equilibrium-plus-conservation overshoot case (:131-234): A_aq -> P
    (k = 1e3), A_aq held at K_eq = 10 times A_gas, and A_aq + P + A_gas = 1e-6
    replacing A_gas's row; absolute tolerances 1e-8 for the two A species,
    1e-12 for P."""
    m = Mechanism(species=["A_gas", "A_aq", "P"], reactions=[], name="overshoot_equilibrium", reorder_state=False,
                  absolute_tolerance=np.array([1e-8, 1e-8, 1e-12]), relative_tolerance=1e-6)
    m.add(arrhenius(A=1.0e3), [1], [(2, 1.0)])
    m.constraints.append(equilibrium_constraint(1, [(0, 1.0)], [(1, 1.0)], K_HLC_ref=10.0, delta_H=0.0,
                                                name="gas_aq_eq"))
    m.constraints.append(linear_constraint(0, [(1, 1.0), (2, 1.0), (0, 1.0)], 1.0e-6, name="mass_conservation"))
    return m


def overshoot_equilibrium_inputs():
    a_gas = 1.0e-6 / 11.0
    return dict(temperature=np.array([298.0]), pressure=np.array([101325.0]),
                air_density=ideal_air_density(np.array([101325.0]), np.array([298.0])),
                concentrations=np.array([[a_gas, 10.0 * a_gas, 0.0]]), custom_params=np.zeros((1, 0)))


def cascade(balance_atol, k, K1, K2):
    """micm's algebraic-error cascade (test/integration/
    test_dae_algebraic_error_insensitivity.cpp:43-170): B_aq -> P with rate k,
    A_aq = K1 A_gas and B_aq = K2 A_aq held by equilibrium constraints, and
    A_aq + B_aq + P + A_gas = 1e-6 replacing A_gas's row; A_gas's absolute
    tolerance is `balance_atol`.  Returns (mechanism, consistent inputs)."""
    m = Mechanism(species=["A_gas", "A_aq", "B_aq", "P"], reactions=[], name="cascade", reorder_state=False,
                  absolute_tolerance=np.array([balance_atol, 1e-8, 1e-8, 1e-12]), relative_tolerance=1e-6)
    m.add(arrhenius(A=k), [2], [(3, 1.0)])
    m.constraints.append(equilibrium_constraint(1, [(0, 1.0)], [(1, 1.0)], K_HLC_ref=K1, delta_H=0.0, name="eq1"))
    m.constraints.append(equilibrium_constraint(2, [(1, 1.0)], [(2, 1.0)], K_HLC_ref=K2, delta_H=0.0, name="eq2"))
    m.constraints.append(linear_constraint(0, [(1, 1.0), (2, 1.0), (3, 1.0), (0, 1.0)], 1.0e-6, name="mass"))
    ag0 = 1.0e-6 / (1.0 + K1 + K1 * K2)
    inputs = dict(temperature=np.array([298.0]), pressure=np.array([101325.0]),
                  air_density=ideal_air_density(np.array([101325.0]), np.array([298.0])),
                  concentrations=np.array([[ag0, K1 * ag0, K2 * K1 * ag0, 0.0]]), custom_params=np.zeros((1, 0)))
    return m, inputs
