"""Classic stiff problems as micm's integration tests set them up.

Robertson's stiff chemical kinetics problem (test/integration/analytical_policy.hpp:1380-1536: A -> B (0.04),
B + B -> B + C (3e7), B + C -> A + C (1e4), air density 1e6, relative
tolerance 1e-10, absolute 1e-12, outputs at t = 1, 10, ..., 1e11).  micm's
test checks micm against a published reference solution; here the C
restatement follows micm itself at every output (identical accepted-step
counts, values within rtol 1e-6), and the GPU follows the restatement exactly.

At rtol 1e-10 over hundreds of steps the step sequence is sensitive to the
last bit of the step-size factor pow(error, 1/order): glibc's pow rounds
wrongly in about one call in a thousand, the GPU's pow (and the restatement's
correctly rounded mode) round correctly.  So the GPU equals the restatement in
its correctly rounded mode bit for bit, accepted-step counts and values at
every output; against micm it meets the criterion micm's own CUDA
Robertson test uses (values within rtol 1e-6 at every output,
test/integration/cuda/test_cuda_analytical_rosenbrock.cpp:185-196), with the
number of outputs at identical step counts recorded.  Tableaus that cover every
output interval within micm's 1,000 steps per Solve: the 4-stage and the
6-stage DA ones (with the others micm runs out of steps in some interval and
calls Solve again)."""
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


def restatement_outputs(tableau, correctly_rounded):
    R = oracle.Restatement(robertson(), tableau_kind=tableau, correctly_rounded=correctly_rounded)
    inp = robertson_inputs()
    out = []
    for dt in intervals():
        y, st = R.solve_per_cell(inp, dt, threads=1)
        inp = dict(inp, concentrations=y)
        out.append((y[0].copy(), int(st[0, 3])))
    return out


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("tableau", [4, 60])
def test_correctly_rounded_restatement_follows_micm(tableau):
    """Only the last bits of pow separate the two modes: values within rtol
    1e-6 at every output, step counts identical at most outputs."""
    cr = restatement_outputs(tableau, True)
    same = 0
    for (y, acc), (y_micm, acc_micm) in zip(cr, micm_outputs(tableau)):
        np.testing.assert_allclose(y, y_micm, rtol=1e-6, atol=1e-30)
        same += acc == acc_micm
    assert same >= 10


@pytest.mark.gpu
@pytest.mark.parametrize("tableau", [4, 60])
@pytest.mark.parametrize("method,step_control", [("plain", "global"), ("fused", "per_cell")])
def test_gpu_equals_correctly_rounded_restatement(cuda_device, tableau, method, step_control):
    from micm_b200 import Solver
    from gpu_helpers import make_state
    solver = Solver(robertson(), tableau, vector_length=1)
    st = make_state(solver, robertson_inputs())
    solver.update_state_parameters(st)
    for dt, (y_ref, acc) in zip(intervals(), restatement_outputs(tableau, True)):
        res = solver.solve(dt, st, method=method, step_control=step_control)
        assert res.converged and res.stats["accepted"] == acc
        st.sync_outputs_to_host()
        np.testing.assert_array_equal(st.concentrations()[0], y_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("tableau", [4, 60])
def test_gpu_follows_micm(cuda_device, tableau):
    from micm_b200 import Solver
    from gpu_helpers import make_state
    solver = Solver(robertson(), tableau, vector_length=1)
    st = make_state(solver, robertson_inputs())
    solver.update_state_parameters(st)
    same = 0
    for dt, (y_micm, acc) in zip(intervals(), micm_outputs(tableau)):
        res = solver.solve(dt, st, method="fused", step_control="per_cell")
        assert res.converged
        same += res.stats["accepted"] == acc
        st.sync_outputs_to_host()
        np.testing.assert_allclose(st.concentrations()[0], y_micm, rtol=1e-6, atol=1e-30)
    assert same >= 10


# ---------------------------------------------------------------------------
# E5 (analytical_policy.hpp TestAnalyticalE5 :2018-: A1 -> A2 + A3 (7.89e-10),
# A2 + A3 -> A5 (1.13e9), A1 + A3 -> A4 (1.1e7), A4 -> A3 + A6 (1.13e3);
# relative tolerance 1e-13, absolute 1e-17 (1e-7 for A1, A5, A6); outputs at
# t = 10, 1e3, ..., 1e13).  micm's test checks micm against a published
# reference solution; the restatement is checked against micm itself.
# Tableaus that cover every output interval within micm's 1,000 steps per
# Solve: 3-stage, 4-stage and both DA ones.
# ---------------------------------------------------------------------------
def e5():
    atol = np.full(6, 1e-17)
    atol[[0, 4, 5]] = 1e-7
    m = Mechanism(species=["A1", "A2", "A3", "A4", "A5", "A6"], reactions=[], name="e5", reorder_state=False,
                  absolute_tolerance=atol, relative_tolerance=1e-13)
    m.add(user_defined("r1"), [0], [(1, 1.0), (2, 1.0)])
    m.add(user_defined("r2"), [1, 2], [(4, 1.0)])
    m.add(user_defined("r3"), [0, 2], [(3, 1.0)])
    m.add(user_defined("r4"), [3], [(2, 1.0), (5, 1.0)])
    return m


def e5_inputs():
    return dict(temperature=np.array([272.5]), pressure=np.array([101253.3]), air_density=np.array([1.0]),
                concentrations=np.array([[1.76e-3, 0.0, 0.0, 0.0, 0.0, 0.0]]),
                custom_params=np.array([[7.89e-10, 1.13e9, 1.1e7, 1.13e3]]))


def e5_intervals():
    t, target = 0.0, 10.0
    for _ in range(7):
        yield target - t
        t, target = target, target * 100


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("tableau", [3, 4, 40, 60])
def test_e5_restatement_follows_micm(tableau):
    ref = oracle.Reference(e5(), tableau=tableau)
    R = oracle.Restatement(e5(), tableau_kind=tableau)
    inp_ref, inp = e5_inputs(), e5_inputs()
    for dt in e5_intervals():
        y_micm, st_micm = ref.solve_global(inp_ref, dt)
        assert st_micm[0]["state"] == 2 and st_micm[0]["final_time"] == dt
        y, st = R.solve_per_cell(inp, dt, threads=1)
        assert st[0, 3] == st_micm[0]["accepted"]
        np.testing.assert_allclose(y, y_micm, rtol=1e-6, atol=1e-30)
        inp_ref, inp = dict(inp_ref, concentrations=y_micm), dict(inp, concentrations=y)


@pytest.mark.gpu
@pytest.mark.parametrize("tableau", [3, 4, 40, 60])
def test_e5_gpu_equals_correctly_rounded_restatement(cuda_device, tableau):
    from micm_b200 import Solver
    from gpu_helpers import make_state
    R = oracle.Restatement(e5(), tableau_kind=tableau, correctly_rounded=True)
    solver = Solver(e5(), tableau, vector_length=1)
    st = make_state(solver, e5_inputs())
    solver.update_state_parameters(st)
    inp = e5_inputs()
    for dt in e5_intervals():
        y_ref, st_ref = R.solve_per_cell(inp, dt, threads=1)
        inp = dict(inp, concentrations=y_ref)
        res = solver.solve(dt, st, method="fused", step_control="per_cell")
        assert res.converged and res.stats["accepted"] == st_ref[0, 3]
        st.sync_outputs_to_host()
        np.testing.assert_array_equal(st.concentrations()[0], y_ref[0])
