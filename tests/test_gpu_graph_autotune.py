"""CUDA-graph replay (micmb_solve_graph) and the autotuner (micmb_autotune)."""
import numpy as np
import pytest

from micm_b200 import Solver, synthetic
from micm_b200.solver import CONVERGED

from gpu_helpers import make_state

pytestmark = pytest.mark.gpu


def test_graph_replay_equals_repeated_solves(cuda_device):
    """n x (UpdateStateParameters + fused Solve) from a CUDA graph gives the
    same bits as n eager calls."""
    cfg = synthetic.CONFIGS["c210"]
    mech = cfg["mech"]()
    inputs = synthetic.cell_inputs(mech, 300, 17, **cfg["inputs"])
    outs = []
    for graph in (False, True):
        solver = Solver(mech, cfg["stages"], vector_length=32)
        st = make_state(solver, inputs)
        if graph:
            solver.solve_graph(60.0, st, 3)  # eager first repeat, then capture and replay
            solver.solve_graph(60.0, st, 2)  # replays the captured graph
        else:
            for _ in range(5):
                solver.update_state_parameters(st)
                solver.solve(60.0, st, method="fused", step_control="per_cell")
        st.sync_outputs_to_host()
        outs.append(st.concentrations())
    np.testing.assert_array_equal(outs[0], outs[1])


def test_autotune_keeps_state_and_caches(cuda_device, tmp_path):
    cfg = synthetic.CONFIGS["c210"]
    mech = cfg["mech"]()
    inputs = synthetic.cell_inputs(mech, 500, 19, **cfg["inputs"])
    solver = Solver(mech, cfg["stages"], vector_length=32)
    st = make_state(solver, inputs)
    solver.update_state_parameters(st)
    cache = str(tmp_path / "tune.txt")
    chosen = solver.autotune(cfg["dt"], st, cache)
    # the state's inputs are restored: a solve now equals a solve on a fresh state
    solver.solve(cfg["dt"], st, method="fused", step_control="per_cell")
    st.sync_outputs_to_host()
    fresh = Solver(mech, cfg["stages"], vector_length=32)
    fresh.set_fused_config(**chosen)
    st2 = make_state(fresh, inputs)
    fresh.update_state_parameters(st2)
    fresh.solve(cfg["dt"], st2, method="fused", step_control="per_cell")
    st2.sync_outputs_to_host()
    np.testing.assert_array_equal(st.concentrations(), st2.concentrations())
    # the cache answers without timing again
    other = Solver(mech, cfg["stages"], vector_length=32)
    st3 = make_state(other, inputs)
    assert other.autotune(cfg["dt"], st3, cache) == chosen
    with open(cache) as f:
        assert len(f.read().splitlines()) == 1


def test_solve_after_autotune_on_more_cells_than_the_trial(cuda_device):
    """The autotuner times a prefix of the state; per-cell outputs of the
    following full solve must still cover every cell."""
    cfg = synthetic.CONFIGS["c210"]
    mech = cfg["mech"]()
    n = 20000  # more than the autotuner's prefix (SMs x 96 cells)
    inputs = synthetic.cell_inputs(mech, n, 23, **cfg["inputs"])
    solver = Solver(mech, cfg["stages"], vector_length=128)
    st = make_state(solver, inputs)
    solver.update_state_parameters(st)
    solver.autotune(60.0, st)
    res = solver.solve(60.0, st, method="fused", step_control="per_cell", per_cell=True)
    assert res.converged
    assert len(res.per_cell_status) == n and np.all(res.per_cell_status == CONVERGED)
