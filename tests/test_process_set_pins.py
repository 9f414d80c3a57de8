"""Forcing and -J against the hand-computed values of micm's ProcessSet test
(test/unit/process/test_process_set_policy.hpp:26-186): six species (corge
unused), a parameterized third body qux (c_rho = 0.72), four Arrhenius
reactions whose rate constants are given with the third body folded in,
two cells, forcing starting at 1000 and the Jacobian at 100.  micm checks
within 4 ULP (1e-12 relative where terms cancel); the restated sums here
start from the fill value in another order, so 1e-13 relative."""
import numpy as np
import pytest

import oracle
from micm_b200.mechanism import Mechanism, arrhenius

RTOL = 1e-13
Y = np.array([[0.1, 0.2, 0.3, 0.4, 0.5, 0.0], [1.1, 1.2, 1.3, 1.4, 1.5, 0.0]])
RHO = np.array([70.0, 80.0])
K = np.array([[10.0, 20.0 * 70.0 * 0.72, 30.0, 40.0 * 70.0 * 0.72],
              [110.0, 120.0 * 80.0 * 0.72, 130.0, 140.0 * 80.0 * 0.72]])


def mechanism():
    foo, bar, baz, quz, quuz = 0, 1, 2, 3, 4
    qux = -1                                   # parameterized reactant 0
    m = Mechanism(species=["foo", "bar", "baz", "quz", "quuz", "corge"], reactions=[], name="process_set",
                  parameterized=[(0.0, 0.0, 0.0, 0.72)], reorder_state=False)
    rate = arrhenius(A=12.2, C=300.0)
    m.add(rate, [foo, baz], [(bar, 1.0), (quuz, 2.4)])
    m.add(rate, [bar, qux], [(foo, 1.0), (quz, 1.4)])
    m.add(rate, [quz], [])
    m.add(rate, [baz, qux], [(bar, 1.0), (quz, 2.5)])
    return m


def expected_forcing():
    f = np.empty((2, 5))
    for c, (y, k) in enumerate(zip(Y, K)):
        foo, bar, baz, quz = y[0], y[1], y[2], y[3]
        f[c, 0] = 1000.0 - k[0] * foo * baz + k[1] * bar
        f[c, 1] = 1000.0 + k[0] * foo * baz - k[1] * bar + k[3] * baz
        f[c, 2] = 1000.0 - k[0] * foo * baz - k[3] * baz
        f[c, 3] = 1000.0 + k[1] * bar * 1.4 - k[2] * quz + k[3] * 2.5 * baz
        f[c, 4] = 1000.0 + k[0] * foo * baz * 2.4
    return f


def expected_jacobian():
    """{(row, col): [cell 0, cell 1]} as listed in the micm test."""
    out = {}
    for c, (y, k) in enumerate(zip(Y, K)):
        foo, baz = y[0], y[2]
        vals = {(0, 0): 100.0 + k[0] * baz, (0, 1): 100.0 - k[1], (0, 2): 100.0 + k[0] * foo,
                (1, 0): 100.0 - k[0] * baz, (1, 1): 100.0 + k[1], (1, 2): 100.0 - k[0] * foo - k[3],
                (2, 0): 100.0 + k[0] * baz, (2, 2): 100.0 + k[0] * foo + k[3],
                (3, 1): 100.0 - 1.4 * k[1], (3, 2): 100.0 - 2.5 * k[3], (3, 3): 100.0 + k[2],
                (4, 0): 100.0 - 2.4 * k[0] * baz, (4, 2): 100.0 - 2.4 * k[0] * foo}
        for key, v in vals.items():
            out.setdefault(key, [0.0, 0.0])[c] = v
    return out


def test_expected_values_restate_micm():
    # spot checks of the restatement against the micm test's own expressions
    f, j = expected_forcing(), expected_jacobian()
    assert f[0, 0] == pytest.approx(1000.0 - 10.0 * 0.1 * 0.3 + 20.0 * 70.0 * 0.72 * 0.2, rel=1e-15)
    assert f[1, 3] == pytest.approx(1000.0 + 120.0 * 80.0 * 0.72 * 1.2 * 1.4 - 130.0 * 1.4
                                    + 140.0 * 80.0 * 0.72 * 2.5 * 1.3, rel=1e-15)
    assert j[(1, 2)][0] == pytest.approx(100.0 - 10.0 * 0.1 - 40.0 * 70.0 * 0.72, rel=1e-15)


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_flattened_description_gives_micm_values():
    ref = oracle.Reference(mechanism(), tableau=3)
    np.testing.assert_array_equal(ref.species_columns, np.arange(6))
    f = ref.forcing(K, Y)
    np.testing.assert_allclose(1000.0 + f[:, :5], expected_forcing(), rtol=RTOL)
    jac = ref.jacobian(K, Y)
    for (r, c), v in expected_jacobian().items():
        e = int(np.nonzero((ref.rows == r) & (ref.cols == c))[0][0])
        np.testing.assert_allclose(100.0 + jac[:, e], v, rtol=RTOL)


@pytest.mark.gpu
def test_gpu_kernels_give_micm_values(cuda_device):
    from micm_b200 import Solver
    from micm_b200 import solver as sv
    from micm_b200._native import check, lib
    from gpu_helpers import download_cols, make_state, upload_cols
    mech = mechanism()
    solver = Solver(mech, 3, vector_length=2)
    inputs = dict(temperature=np.array([298.15, 298.15]), pressure=np.array([101325.0, 101325.0]),
                  air_density=RHO, concentrations=Y, custom_params=np.zeros((2, 0)))
    st = make_state(solver, inputs)
    np.testing.assert_array_equal(solver.compiled.species_columns, np.arange(6))
    upload_cols(st, sv.BUF_RATE_CONSTANTS, K)
    upload_cols(st, sv.BUF_VARIABLES, Y)
    upload_cols(st, sv.BUF_FORCING, np.full((2, 6), 1000.0))
    check(lib().micmb_add_forcing_terms(solver.handle, st.handle))
    f = download_cols(st, sv.BUF_FORCING, 6)
    np.testing.assert_allclose(f[:, :5], expected_forcing(), rtol=RTOL)
    rows, cols = solver.compiled.rows, solver.compiled.cols
    upload_cols(st, sv.BUF_JACOBIAN, np.full((2, len(rows)), 100.0))
    check(lib().micmb_subtract_jacobian_terms(solver.handle, st.handle))
    jac = download_cols(st, sv.BUF_JACOBIAN, len(rows))
    for (r, c), v in expected_jacobian().items():
        e = int(np.nonzero((rows == r) & (cols == c))[0][0])
        np.testing.assert_allclose(jac[:, e], v, rtol=RTOL)
