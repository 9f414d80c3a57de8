"""Backward Euler (micm's second integrator: include/micm/solver/backward_euler.inl,
default parameters) restated in the C oracle, as the checker for a GPU
Backward Euler built on the same forcing, -J, LU and solve kernels.  Pinned
two ways: bit for bit against micm's own Backward Euler (oracle/_ref, in-place
Mozart LU, a 1-cell State per cell) including the solver statistics, the
rejection and step-doubling paths and the unconverged-acceptance path; and
against micm's flow-tube regression golden for Backward Euler
(test/regression/expected_results/backward_euler_wall_loss.csv, all 3,601 rows
within the file's 6 significant digits)."""
import os

import numpy as np
import pytest

import oracle
from micm_b200 import micm_bench, synthetic

from test_flow_tube import flow_tube, flow_tube_inputs

pytestmark = pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
GOLDEN = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "backward_euler_wall_loss.npz"))


def test_reproduces_micms_flow_tube_golden():
    R = oracle.Restatement(flow_tube(), tableau_kind=2)
    inp = flow_tube_inputs()
    out = [inp["concentrations"][0]]
    for _ in range(3600):
        y, stats = R.backward_euler_per_cell(inp, 1.0)
        assert stats[0, 7] == 2
        inp = dict(inp, concentrations=y)
        out.append(y[0])
    np.testing.assert_allclose(np.array(out), GOLDEN["concentrations"], rtol=1e-5, atol=1e-20)


CASES = [
    # (mechanism, inputs, dt): one step; rejections, reductions and doubling; micm_bench's mechanisms
    ("syn60_600", lambda: synthetic.synthetic_mechanism(60, 120, seed=601), lambda m: synthetic.cell_inputs(m, 32, 5), 600.0),
    ("syn60_3600", lambda: synthetic.synthetic_mechanism(60, 120, seed=601), lambda m: synthetic.cell_inputs(m, 32, 5), 3600.0),
    ("syn60_1day", lambda: synthetic.synthetic_mechanism(60, 120, seed=601), lambda m: synthetic.cell_inputs(m, 32, 5), 86400.0),
    ("chapman", lambda: micm_bench.mechanism("chapman"), lambda m: micm_bench.inputs("chapman", 16, seed=3), 30.0),
    # TS1 at dt = 30 s: Newton fails five times and micm accepts the unconverged step
    ("ts1_unconverged", lambda: micm_bench.mechanism("ts1", absolute_tolerance=1e-9),
     lambda m: micm_bench.inputs("ts1", 4, seed=3), 30.0),
]


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,make_mech,make_inputs,dt", CASES, ids=[c[0] for c in CASES])
def test_equals_micms_backward_euler(name, make_mech, make_inputs, dt):
    mech = make_mech()
    inp = make_inputs(mech)
    y, stats = oracle.Restatement(mech, tableau_kind=3).backward_euler_per_cell(inp, dt)
    y_micm, stats_micm = oracle.Reference(mech, tableau=3).backward_euler_per_cell(inp, dt)
    np.testing.assert_array_equal(y, y_micm)
    np.testing.assert_array_equal(stats[:, :9], stats_micm[:, :9])     # counters, state, final time
    if name == "syn60_1day":
        assert stats[:, 4].max() >= 3 and stats[:, 3].max() >= 5     # rejections and several accepted steps
    if name == "ts1_unconverged":
        assert np.all(stats[:, 7] == 8)                                # AcceptingUnconvergedIntegration


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,make_mech,make_inputs,dt", CASES, ids=[c[0] for c in CASES])
def test_global_equals_micms_multi_cell_backward_euler(name, make_mech, make_inputs, dt):
    """micm's n-cell State (one step size, one convergence test over all cells)."""
    mech = make_mech()
    inp = make_inputs(mech)
    y, stats = oracle.Restatement(mech, tableau_kind=3).backward_euler_global(inp, dt)
    y_micm, stats_micm = oracle.Reference(mech, tableau=3).backward_euler_global(inp, dt)
    np.testing.assert_array_equal(y, y_micm)
    np.testing.assert_array_equal(stats[:9], stats_micm[:9])
