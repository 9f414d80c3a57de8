"""Helpers for GPU parity tests."""
import numpy as np

from micm_b200 import Solver
from micm_b200.mechanism import from_vector_layout, padded_cells, to_vector_layout
from micm_b200 import solver as sv


def make_state(solver: Solver, inputs, L=None):
    n = len(inputs["temperature"])
    st = solver.get_state(n, L)
    st.set_inputs(inputs)
    st.sync_inputs_to_device()
    return st


def upload_cols(st, buf, a):
    st.upload(buf, to_vector_layout(np.asarray(a, dtype=np.float64), st.L))


def download_cols(st, buf, ncols):
    npad = padded_cells(st.n_cells, st.L)
    return from_vector_layout(st.download(buf, npad * ncols), st.n_cells, ncols, st.L)


def solve_gpu(mech, inputs, dt, stages, method, step_control, n_solves=1, L=32, fused_config=None):
    solver = Solver(mech, stages, vector_length=L)
    if fused_config:
        solver.set_fused_config(**fused_config)
    st = make_state(solver, inputs)
    results = []
    for _ in range(n_solves):
        solver.update_state_parameters(st)
        results.append(solver.solve(dt, st, method=method, step_control=step_control, per_cell=True))
    st.sync_outputs_to_host()
    return st.concentrations(), results
