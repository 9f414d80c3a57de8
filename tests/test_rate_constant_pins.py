"""Rate constants against the known answers of micm's own rate-constant unit
tests (test/unit/process/rate_constant/test_*_rate_constant.cpp): each case
is a one-reaction mechanism evaluated at the test's conditions, the expected
value restated from the test's formula.  The C restatement is checked on the
CPU within micm's tolerances (1e-13 relative; 1e-14 where micm asserts exact
equality of the same formula in another operation order), the GPU kernel
within 1e-12 (CUDA's exp/pow/log10 differ from the host library in the last
bits)."""
import math

import numpy as np
import pytest

import oracle
from micm_b200.mechanism import (AVOGADRO_CONSTANT, GAS_CONSTANT, Mechanism, arrhenius, branched, reversible,
                                 surface, taylor_series, ternary, troe, tunneling, user_defined)

T0, RHO = 301.24, 42.2


def _fc_power(fc, n, x):
    return math.pow(fc, n / (n + math.pow(math.log10(x), 2)))


def _falloff_k(A, B, C, T):
    return A * math.exp(C / T) * math.pow(T / 300.0, B)


def _branched_expected(branch, X, Y, a0, n, T, rho):
    # test_branched_rate_constant.cpp: z from the reference air density 2.45e19 molec cm-3 at 293 K
    a = 2.0e-22 * math.exp(n) * 2.45e19
    b = 0.43 * math.pow(293.0 / 298.0, -8.0)
    z = a / (1.0 + a / b) * math.pow(0.41, 1.0 / (1.0 + math.pow(math.log10(a / b), 2))) * (1.0 - a0) / a0
    a = 2.0e-22 * math.exp(n) * rho * AVOGADRO_CONSTANT * 1.0e-6
    b = 0.43 * math.pow(T / 298.0, -8.0)
    A = a / (1.0 + a / b) * math.pow(0.41, 1.0 / (1.0 + math.pow(math.log10(a / b), 2)))
    pre = X * math.exp(-Y / T)
    return pre * (z / (z + A)) if branch == 0 else pre * (A / (z + A))


def _surface_expected(D, mw, gamma, T, radius, number):
    speed = math.sqrt(8.0 * GAS_CONSTANT * T / (math.pi * mw))
    return 4.0 * number * math.pi * radius ** 2 / (radius / D + 4.0 / (speed * gamma))


# (id, rate, temperature, air density, custom parameters, expected, relative tolerance on the CPU)
CASES = [
    # test_arrhenius_rate_constant.cpp:13-50
    ("arrhenius_default", arrhenius(), T0, RHO, [], 1.0, 1e-13),
    ("arrhenius_A", arrhenius(A=2.2e-10), T0, RHO, [], 2.2e-10, 1e-13),
    ("arrhenius_O_HO2", arrhenius(A=3e-11, C=-200.0), T0, RHO, [], 3e-11 * math.exp(-200 / 301.24), 1e-13),
    ("arrhenius_OH_HCl", arrhenius(A=2.6e-12, C=-350.0), T0, RHO, [], 2.6e-12 * math.exp(-350 / 301.24), 1e-13),
    # test_troe_rate_constant.cpp:13-50 (the test asserts exact equality with its own formula)
    ("troe_minimal", troe(k0_A=1.0, kinf_A=1.0), T0, RHO, [],
     RHO * 1.0 / (1.0 + RHO * 1.0 / 1.0) * _fc_power(0.6, 1.0, RHO * 1.0 / 1.0), 1e-14),
    ("troe_all", troe(1.2, 2.3, 302.3, 2.6, -3.1, 402.1, 0.9, 1.2), T0, RHO, [],
     (lambda k0, ki: RHO * k0 / (1.0 + RHO * k0 / ki) * _fc_power(0.9, 1.2, RHO * k0 / ki))(
         _falloff_k(1.2, 2.3, 302.3, T0), _falloff_k(2.6, -3.1, 402.1, T0)), 1e-14),
    ("troe_analytical_BC", troe(1.2e-12, 167.0, 3.0, 136.0, 5.0, 24.0, 0.9, 0.8), T0, RHO, [],
     (lambda k0, ki: k0 * RHO / (1.0 + k0 * RHO / ki) * _fc_power(0.9, 0.8, k0 * RHO / ki))(
         _falloff_k(1.2e-12, 167.0, 3.0, T0), _falloff_k(136.0, 5.0, 24.0, T0)), 1e-14),
    # test_ternary_chemical_activation_rate_constant.cpp:13-50
    ("ternary_minimal", ternary(k0_A=1.0, kinf_A=1.0), T0, RHO, [],
     1.0 / (1.0 + 1.0 * RHO / 1.0) * _fc_power(0.6, 1.0, 1.0 * RHO / 1.0), 1e-14),
    ("ternary_all", ternary(1.2, 2.3, 302.3, 2.6, -3.1, 402.1, 0.9, 1.2), T0, RHO, [],
     (lambda k0, ki: k0 / (1.0 + RHO * k0 / ki) * _fc_power(0.9, 1.2, RHO * k0 / ki))(
         _falloff_k(1.2, 2.3, 302.3, T0), _falloff_k(2.6, -3.1, 402.1, T0)), 1e-14),
    # test_tunneling_rate_constant.cpp:13-35
    ("tunneling_default", tunneling(), T0, RHO, [], 1.0, 1e-13),
    ("tunneling_all", tunneling(A=1.2, B=2.3, C=302.3), T0, RHO, [],
     1.2 * math.exp(-2.3 / T0) * math.exp(302.3 / math.pow(T0, 3)), 1e-13),
    # test_reversible_rate_constant.cpp
    ("reversible_default", reversible(), 298.15, RHO, [], 0.0, 0.0),
    ("reversible_301", reversible(A=1.14e-2, C=2300.0, k_r=0.32), T0, RHO, [],
     1.14e-2 * math.exp(2300.0 / 301.24) * 0.32, 1e-13),
    ("reversible_298", reversible(A=1.14e-2, C=2300.0, k_r=0.32), 298.15, RHO, [],
     1.14e-2 * math.exp(2300.0 / 298.15) * 0.32, 1e-13),
] + [(f"reversible_T{T}", reversible(A=1.5, C=2000.0, k_r=0.5), T, RHO, [], 1.5 * math.exp(2000.0 / T) * 0.5, 1e-13)
     for T in (273.15, 298.15, 323.15)] + [
    # test_taylor_series_rate_constant.cpp:13-50
    ("taylor_default", taylor_series(), T0, RHO, [], 1.0, 1e-13),
    ("taylor_O_HO2", taylor_series(A=3e-11, C=-200.0, coefficients=(12.5, 1.3e-2, 5.2e-4)), T0, RHO, [],
     3e-11 * math.exp(-200 / 301.24) * (12.5 + 1.3e-2 * 301.24 + 5.2e-4 * math.pow(301.24, 2)), 1e-13),
    ("taylor_OH_HCl", taylor_series(A=2.6e-12, C=-350.0, coefficients=(1.0, 4.3e-1, 7.3e-3)), T0, RHO, [],
     2.6e-12 * math.exp(-350 / 301.24) * (1.0 + 4.3e-1 * 301.24 + 7.3e-3 * math.pow(301.24, 2)), 1e-13),
    # test_branched_rate_constant.cpp (alkoxy and nitrate branches)
    ("branched_alkoxy", branched(0, 1.2, 204.3, 1.0e-3, 2), T0, RHO, [],
     _branched_expected(0, 1.2, 204.3, 1.0e-3, 2, T0, RHO), 1e-13),
    ("branched_nitrate", branched(1, 1.2, 204.3, 1.0e-3, 2), T0, RHO, [],
     _branched_expected(1, 1.2, 204.3, 1.0e-3, 2, T0, RHO), 1e-13),
    # test_user_defined_rate_constant.cpp
    ("user_defined", user_defined("foo"), T0, RHO, [0.5], 0.5, 0.0),
    ("user_defined_scaled", user_defined("foo", scaling_factor=2.0), T0, RHO, [1.2], 1.2 * 2.0, 1e-15),
    # test_surface_rate_constant.cpp:13-68 (radius 1e-7 m, 2.5e6 particles m-3)
    ("surface_default_probability", surface("foo", 2.3e2, 0.025), 273.65, RHO, [1.0e-7, 2.5e6],
     _surface_expected(2.3e2, 0.025, 1.0, 273.65, 1.0e-7, 2.5e6), 1e-13),
    ("surface_probability", surface("foo", 2.3e2, 0.025, 0.74), 273.65, RHO, [1.0e-7, 2.5e6],
     _surface_expected(2.3e2, 0.025, 0.74, 273.65, 1.0e-7, 2.5e6), 1e-13),
]


def _mechanism(rate):
    m = Mechanism(species=["A", "B"], reactions=[], name="pin")
    m.add(rate, [0], [(1, 1.0)])
    return m


def _inputs(T, rho, params):
    return dict(temperature=np.array([T]), pressure=np.array([101325.0]), air_density=np.array([rho]),
                concentrations=np.array([[1.0, 0.0]]), custom_params=np.array([params], dtype=np.float64).reshape(1, -1))


def _check(k, expected, rtol):
    if expected == 0.0:
        assert k == 0.0
    else:
        assert abs(k - expected) <= rtol * abs(expected), (k, expected)


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("name,rate,T,rho,params,expected,rtol", CASES, ids=[c[0] for c in CASES])
def test_restatement_matches_micm_unit_tests(name, rate, T, rho, params, expected, rtol):
    R = oracle.Restatement(_mechanism(rate), tableau_kind=3)
    inp = _inputs(T, rho, params)
    k = R.rate_constants(inp["temperature"], inp["pressure"], inp["air_density"], inp["custom_params"])
    _check(float(k[0, 0]), expected, rtol)


@pytest.mark.gpu
@pytest.mark.parametrize("name,rate,T,rho,params,expected,rtol", CASES, ids=[c[0] for c in CASES])
def test_gpu_matches_micm_unit_tests(cuda_device, name, rate, T, rho, params, expected, rtol):
    from micm_b200 import Solver
    from gpu_helpers import make_state
    solver = Solver(_mechanism(rate), 3, vector_length=1)
    st = make_state(solver, _inputs(T, rho, params))
    solver.update_state_parameters(st)
    _check(float(st.rate_constants()[0, 0]), expected, max(rtol, 1e-12))
