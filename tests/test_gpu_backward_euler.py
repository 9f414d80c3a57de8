"""Backward Euler on the GPU (micm's second integrator,
include/micm/solver/backward_euler.inl:10-246, default parameters) against the
C restatement of micm's algorithm, which the CPU tests pin bit for bit to
micm's own Backward Euler (tests/test_backward_euler.py).

With the restatement's rate constants uploaded into the state, the GPU's
results equal the restatement's bit for bit, statistics included, in both
forms: per cell (each cell as micm solves a 1-cell State; one persistent
kernel) and global (micm's n-cell State: one step size and one convergence
test for all cells).  The cases cover one-step solves, rejections with
time-step reductions and step doubling, and micm's acceptance of an
unconverged step.  With the GPU's own rate constants the results follow micm
itself, and the flow-tube regression golden for Backward Euler
(test/regression/expected_results/backward_euler_wall_loss.csv) is
reproduced over all 3,600 solves."""
import os

import numpy as np
import pytest

import oracle
from micm_b200 import Solver, micm_bench, synthetic
from micm_b200 import solver as sv

from gpu_helpers import make_state, upload_cols
from test_backward_euler import CASES
from test_flow_tube import flow_tube, flow_tube_inputs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")]
GOLDEN = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "backward_euler_wall_loss.npz"))
STATS = ("function_calls", "jacobian_updates", "number_of_steps", "accepted", "rejected", "decompositions", "solves")


def _gpu(mech, inp, dt, step_control, k=None, L=32):
    solver = Solver(mech, 3, vector_length=L)
    st = make_state(solver, inp)
    if k is None:
        solver.update_state_parameters(st)
    else:
        upload_cols(st, sv.BUF_RATE_CONSTANTS, k)
    res = solver.solve_backward_euler(dt, st, step_control, per_cell=True)
    st.sync_outputs_to_host()
    return st.concentrations(), res


@pytest.mark.parametrize("name,make_mech,make_inputs,dt", CASES, ids=[c[0] for c in CASES])
def test_per_cell_equals_restatement(cuda_device, name, make_mech, make_inputs, dt):
    mech = make_mech()
    inp = make_inputs(mech)
    R = oracle.Restatement(mech, tableau_kind=3)
    k = R._k(inp)
    y_ref, st_ref = R.backward_euler_per_cell(inp, dt, k=k)
    y, res = _gpu(mech, inp, dt, "per_cell", k=k)
    np.testing.assert_array_equal(y, y_ref)
    np.testing.assert_array_equal(res.per_cell_status, st_ref[:, 7])
    np.testing.assert_array_equal(res.per_cell_accepted, st_ref[:, 3])
    for q, key in enumerate(STATS):
        assert res.stats[key] == st_ref[:, q].sum(), key


@pytest.mark.parametrize("name,make_mech,make_inputs,dt", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("L", [1, 32])
def test_global_equals_restatement(cuda_device, name, make_mech, make_inputs, dt, L):
    mech = make_mech()
    inp = make_inputs(mech)
    R = oracle.Restatement(mech, tableau_kind=3)
    k = R._k(inp)
    y_ref, st_ref = R.backward_euler_global(inp, dt, k=k)
    y, res = _gpu(mech, inp, dt, "global", k=k, L=L)
    np.testing.assert_array_equal(y, y_ref)
    for q, key in enumerate(STATS):
        assert res.stats[key] == st_ref[q], key
    assert res.state == st_ref[7]
    assert res.stats["final_time"] == st_ref[8:9].view(np.float64)[0]
    assert np.all(res.per_cell_status == st_ref[7])


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,make_mech,make_inputs,dt", CASES[:4], ids=[c[0] for c in CASES[:4]])
def test_follows_micm_with_own_rate_constants(cuda_device, name, make_mech, make_inputs, dt):
    mech = make_mech()
    inp = make_inputs(mech)
    y_micm, st_micm = oracle.Reference(mech, tableau=3).backward_euler_per_cell(inp, dt)
    y, res = _gpu(mech, inp, dt, "per_cell")
    np.testing.assert_allclose(y, y_micm, rtol=1e-6, atol=1e-12)
    assert np.mean(res.per_cell_accepted == st_micm[:, 3]) >= 0.999


def test_flow_tube_golden(cuda_device):
    solver = Solver(flow_tube(), 3, vector_length=1)
    st = make_state(solver, flow_tube_inputs())
    solver.update_state_parameters(st)
    out = [flow_tube_inputs()["concentrations"][0]]
    for _ in range(3600):
        res = solver.solve_backward_euler(1.0, st, "global")
        assert res.state == 2
        st.sync_outputs_to_host()
        out.append(st.concentrations()[0])
    np.testing.assert_allclose(np.array(out), GOLDEN["concentrations"], rtol=1e-5, atol=1e-20)
