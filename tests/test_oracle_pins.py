"""Pins the checkers to the reference's own published results."""
import numpy as np
import pytest

import oracle
from micm_b200 import synthetic
from micm_b200.mechanism import ideal_air_density

pytestmark = pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")

# README.md:170-182 (three significant digits)
README_TABLE = [
    (1.18e+01, 5.90e+00, 1.91e+00), (6.79e+00, 9.05e+00, 3.32e+00), (3.83e+00, 1.07e+01, 4.21e+00),
    (2.14e+00, 1.17e+01, 4.74e+00), (1.19e+00, 1.22e+01, 5.04e+00), (6.58e-01, 1.24e+01, 5.21e+00),
    (3.64e-01, 1.26e+01, 5.31e+00), (2.01e-01, 1.27e+01, 5.36e+00), (1.11e-01, 1.27e+01, 5.39e+00),
    (6.13e-02, 1.28e+01, 5.41e+00),
]


def test_reference_reproduces_readme_table():
    m = synthetic.readme_mechanism()
    ref = oracle.Reference(m, tableau=3)
    T = np.array([287.45]); P = np.array([101319.9])
    inputs = dict(temperature=T, pressure=P, air_density=ideal_air_density(P, T),
                  concentrations=np.array([[20.0, 0.0, 0.0]]), custom_params=np.zeros((1, 0)))
    for row in README_TABLE:
        y, _ = ref.solve_global(inputs, 500.0)
        inputs["concentrations"] = y
        assert [float(f"{v:.2e}") for v in y[0]] == list(row)


def test_reference_matches_abc_closed_form():
    """A -k1-> B -k2-> C against its closed form (test/integration/analytical_policy.hpp:138-276)."""
    m = synthetic.abc_mechanism()
    ref = oracle.Reference(m, tableau=4)
    T = np.array([272.5, 254.7, 312.6]); P = np.array([101253.3, 100672.5, 101319.8])
    rho = ideal_air_density(P, T)
    k = ref.rate_constants(T, P, rho, np.zeros((3, 1)))
    k1, k2 = k[:, 0], k[:, 1]
    y0 = np.array([[1.0, 0, 0], [2.0 / 3, 0, 0], [1.0 / 3, 0, 0]])
    inputs = dict(temperature=T, pressure=P, air_density=rho, concentrations=y0.copy(), custom_params=np.zeros((3, 0)))
    for step in range(1, 30):
        y, _ = ref.solve_global(inputs, 1.0)
        inputs["concentrations"] = y
        t = float(step)
        A = y0[:, 0] * np.exp(-k1 * t)
        B = y0[:, 0] * (k1 / (k2 - k1)) * (np.exp(-k1 * t) - np.exp(-k2 * t))
        C = y0[:, 0] * (1.0 + (k1 * np.exp(-k2 * t) - k2 * np.exp(-k1 * t)) / (k2 - k1))
        np.testing.assert_allclose(y[:, 0], A, atol=1e-4)
        np.testing.assert_allclose(y[:, 1], B, atol=1e-4)
        np.testing.assert_allclose(y[:, 2], C, atol=1e-4)
