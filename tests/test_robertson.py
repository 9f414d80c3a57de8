"""Robertson's stiff chemical kinetics problem as micm's integration test sets
it up (test/integration/analytical_policy.hpp:1380-1536: A -> B (0.04),
B + B -> B + C (3e7), B + C -> A + C (1e4), air density 1e6, relative
tolerance 1e-10, absolute 1e-12, outputs at t = 1, 10, ..., 1e11).  micm's
test checks micm against a published reference solution; here the C
restatement and the GPU are checked against micm itself (oracle/_ref) at every
output: identical accepted-step counts, values within rtol 1e-6.  Tableaus
that cover every output interval within micm's 1,000 steps per Solve: the
4-stage and the 6-stage DA ones (with the others micm runs out of steps in
some interval and calls Solve again)."""
import numpy as np
import pytest

import oracle
from micm_b200.mechanism import Mechanism, user_defined

pytestmark = pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")


def robertson():
    m = Mechanism(species=["A", "B", "C"], reactions=[], name="robertson", reorder_state=False,
                  absolute_tolerance=np.full(3, 1e-12), relative_tolerance=1e-10)
    m.add(user_defined("r1"), [0], [(1, 1.0)])
    m.add(user_defined("r2"), [1, 1], [(1, 1.0), (2, 1.0)])
    m.add(user_defined("r3"), [1, 2], [(0, 1.0), (2, 1.0)])
    return m


def robertson_inputs():
    return dict(temperature=np.array([272.5]), pressure=np.array([101253.3]), air_density=np.array([1e6]),
                concentrations=np.array([[1.0, 0.0, 0.0]]), custom_params=np.array([[0.04, 3e7, 1e4]]))


def intervals():
    t, target = 0.0, 1.0
    for _ in range(12):
        yield target - t
        t, target = target, target * 10


def micm_outputs(tableau):
    ref = oracle.Reference(robertson(), tableau=tableau)
    inp = robertson_inputs()
    out = []
    for dt in intervals():
        y, st = ref.solve_global(inp, dt)
        assert st[0]["state"] == 2 and st[0]["final_time"] == dt
        inp = dict(inp, concentrations=y)
        out.append((y[0].copy(), st[0]["accepted"]))
    return out


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("tableau", [4, 60])
def test_restatement_follows_micm(tableau):
    R = oracle.Restatement(robertson(), tableau_kind=tableau)
    inp = robertson_inputs()
    for dt, (y_micm, acc) in zip(intervals(), micm_outputs(tableau)):
        y, st = R.solve_per_cell(inp, dt, threads=1)
        assert st[0, 3] == acc
        np.testing.assert_allclose(y[0], y_micm, rtol=1e-6, atol=1e-30)
        inp = dict(inp, concentrations=y)


@pytest.mark.gpu
@pytest.mark.parametrize("tableau", [4])
@pytest.mark.parametrize("method,step_control", [("plain", "global"), ("fused", "per_cell")])
def test_gpu_follows_micm(cuda_device, tableau, method, step_control):
    from micm_b200 import Solver
    from gpu_helpers import make_state
    solver = Solver(robertson(), tableau, vector_length=1)
    st = make_state(solver, robertson_inputs())
    solver.update_state_parameters(st)
    for dt, (y_micm, acc) in zip(intervals(), micm_outputs(tableau)):
        res = solver.solve(dt, st, method=method, step_control=step_control)
        assert res.converged and res.stats["accepted"] == acc
        st.sync_outputs_to_host()
        np.testing.assert_allclose(st.concentrations()[0], y_micm, rtol=1e-6, atol=1e-30)
