"""micm's flow-tube regression (test/regression/regression_policy.hpp,
TestFlowTube, with the 2-stage Rosenbrock solver of
test/regression/test_regression.cpp): 3,600 Solve(1 s) calls on a
4-species wall-loss mechanism, against micm's stored results
(tests/golden/rosenbrock_wall_loss.npz, from
test/regression/expected_results/rosenbrock_wall_loss.csv).  micm's own test
compares the first 10 rows within 1e-10; here every row is compared within
the file's precision (6 significant digits: rtol 1e-5)."""
import os

import numpy as np
import pytest

import oracle
from micm_b200.mechanism import Mechanism, arrhenius, ideal_air_density, user_defined

GOLDEN = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rosenbrock_wall_loss.npz"))
RTOL, ATOL = 1e-5, 1e-20


def flow_tube():
    """SOA1 -> (r1), SOA2 -> (r2), O3 + a-pinene -> 0.18 SOA1 + 0.09 SOA2 (Arrhenius
    A = 8.8e-17 cm3 molec-1 s-1 in mol m-3 units); micm's default tolerances."""
    m = Mechanism(species=["SOA1", "SOA2", "a-pinene", "O3"], reactions=[], name="flow_tube", reorder_state=False)
    m.add(user_defined("r1"), [0], [])
    m.add(user_defined("r2"), [1], [])
    m.add(arrhenius(A=8.8e-17 * (1.0e-6 * 6.02214076e23)), [2, 3], [(0, 0.18), (1, 0.09)])
    return m


def flow_tube_inputs():
    T, P = np.array([298.15]), np.array([101325.0])
    return dict(temperature=T, pressure=P, air_density=ideal_air_density(P, T),
                concentrations=np.array([[0.0, 0.0, 8e-8, 0.00002]]), custom_params=np.array([[0.01, 0.05]]))


def test_fixture_shape():
    assert list(GOLDEN["species"]) == ["SOA1", "SOA2", "a-pinene", "O3"]
    assert GOLDEN["concentrations"].shape == (3601, 4)
    np.testing.assert_array_equal(GOLDEN["concentrations"][0], flow_tube_inputs()["concentrations"][0])


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
def test_restatement_reproduces_micm_flow_tube():
    R = oracle.Restatement(flow_tube(), tableau_kind=2)
    inp = flow_tube_inputs()
    out = [inp["concentrations"][0]]
    for _ in range(3600):
        y, stats = R.solve_per_cell(inp, 1.0, threads=1)
        assert stats[0, 7] == 2          # converged over the whole second
        inp = dict(inp, concentrations=y)
        out.append(y[0])
    np.testing.assert_allclose(np.array(out), GOLDEN["concentrations"], rtol=RTOL, atol=ATOL)


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["plain", "fused"])
def test_gpu_reproduces_micm_flow_tube(cuda_device, method):
    from micm_b200 import Solver
    from gpu_helpers import make_state
    solver = Solver(flow_tube(), 2, vector_length=1)
    st = make_state(solver, flow_tube_inputs())
    solver.update_state_parameters(st)
    out = [flow_tube_inputs()["concentrations"][0]]
    for _ in range(3600):
        res = solver.solve(1.0, st, method=method, step_control="per_cell")
        assert res.converged
        st.sync_outputs_to_host()
        out.append(st.concentrations()[0].copy())
    np.testing.assert_allclose(np.array(out), GOLDEN["concentrations"], rtol=RTOL, atol=ATOL)
