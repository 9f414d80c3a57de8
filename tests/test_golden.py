"""Parity against committed golden fixtures produced by micm itself
(tests/golden/make_golden.py runs micm's CPU solver, compiled from the
reference sources, on seeded inputs): the CPU restatement on the CPU, the
CUDA kernels and solves on the GPU.  Neither needs the reference at run time."""
import os

import numpy as np
import pytest

import oracle
from micm_b200 import Solver, synthetic
from micm_b200 import solver as sv

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL, ATOL = 1e-6, 1e-12
MECHS = {"syn210": lambda: synthetic.synthetic_mechanism(210, 440, seed=2101),
         "syn60": lambda: synthetic.synthetic_mechanism(60, 120, seed=601)}


def load(name):
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


def inputs_of(g):
    return {k: g[k] for k in ("temperature", "pressure", "air_density", "concentrations", "custom_params") if k in g}


# ---------------------------------------------------------------- CPU: the oracle
@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("name", ["syn210", "syn60"])
def test_restatement_rate_constants_match_micm(name):
    g = load(f"{name}_kernels.npz")
    R = oracle.Restatement(MECHS[name](), tableau_kind=4)
    k = R.rate_constants(g["temperature"], g["pressure"], g["air_density"], g["custom_params"])
    np.testing.assert_allclose(k, g["k"], rtol=1e-14, atol=0)
    np.testing.assert_array_equal(R.species_columns, g["species_columns"])
    np.testing.assert_array_equal(R.rows, g["rows"])
    np.testing.assert_array_equal(R.cols, g["cols"])


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
@pytest.mark.parametrize("name", ["syn210", "syn60"])
def test_restatement_per_cell_solves_match_micm(name):
    g = load(f"{name}_per_cell.npz")
    R = oracle.Restatement(MECHS[name](), tableau_kind=int(g["tableau"]))
    y, stats = R.solve_per_cell(inputs_of(g), float(g["dt"]))
    np.testing.assert_allclose(y, g["y_final"], rtol=RTOL, atol=ATOL)
    np.testing.assert_array_equal(stats[:, 3], g["stats"][:, 3])  # accepted steps per cell


# ---------------------------------------------------------------- GPU: the product
@pytest.mark.gpu
@pytest.mark.parametrize("name,L", [("syn210", 4), ("syn60", 32)])
def test_gpu_kernels_match_micm(cuda_device, name, L):
    from gpu_helpers import download_cols, make_state, upload_cols
    from micm_b200._native import check, lib
    g = load(f"{name}_kernels.npz")
    mech = MECHS[name]()
    n = len(g["temperature"])
    solver = Solver(mech, 4, vector_length=L)
    st = make_state(solver, dict(inputs_of(g), concentrations=np.zeros((n, mech.n_species))))
    solver.update_state_parameters(st)
    np.testing.assert_allclose(st.rate_constants(), g["k"], rtol=1e-12, atol=0)
    upload_cols(st, sv.BUF_RATE_CONSTANTS, g["k"])
    upload_cols(st, sv.BUF_VARIABLES, g["y"])
    upload_cols(st, sv.BUF_FORCING, np.zeros_like(g["y"]))
    check(lib().micmb_add_forcing_terms(solver.handle, st.handle))
    np.testing.assert_array_equal(download_cols(st, sv.BUF_FORCING, mech.n_species), g["forcing"])
    nnz = len(g["rows"])
    upload_cols(st, sv.BUF_JACOBIAN, np.zeros((n, nnz)))
    check(lib().micmb_subtract_jacobian_terms(solver.handle, st.handle))
    np.testing.assert_array_equal(download_cols(st, sv.BUF_JACOBIAN, nnz), g["jacobian"])
    check(lib().micmb_alpha_minus_jacobian(solver.handle, st.handle, float(g["alpha"])))
    check(lib().micmb_lu_decompose(solver.handle, st.handle))
    np.testing.assert_array_equal(download_cols(st, sv.BUF_JACOBIAN, nnz), g["lu"])
    upload_cols(st, sv.BUF_FORCING, g["forcing"])
    check(lib().micmb_linear_solve(solver.handle, st.handle))
    np.testing.assert_array_equal(download_cols(st, sv.BUF_FORCING, mech.n_species), g["x"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["syn210", "syn60"])
@pytest.mark.parametrize("method,config", [("plain", None), ("fused", dict(variant=0)), ("fused", dict(variant=2))])
def test_gpu_per_cell_solves_match_micm(cuda_device, name, method, config):
    from gpu_helpers import make_state
    g = load(f"{name}_per_cell.npz")
    mech = MECHS[name]()
    solver = Solver(mech, int(g["tableau"]), vector_length=32)
    if config:
        solver.set_fused_config(**config)
    st = make_state(solver, inputs_of(g))
    solver.update_state_parameters(st)
    res = solver.solve(float(g["dt"]), st, method=method, step_control="per_cell", per_cell=True)
    st.sync_outputs_to_host()
    np.testing.assert_allclose(st.concentrations(), g["y_final"], rtol=RTOL, atol=ATOL)
    np.testing.assert_array_equal(res.per_cell_accepted, g["stats"][:, 3])


@pytest.mark.gpu
def test_gpu_readme_global_matches_micm(cuda_device):
    from gpu_helpers import make_state
    g = load("readme_global.npz")
    solver = Solver(synthetic.readme_mechanism(), 3, vector_length=4)
    st = make_state(solver, inputs_of(g))
    for i in range(10):
        solver.update_state_parameters(st)
        solver.solve(500.0, st, method="plain", step_control="global")
        st.sync_outputs_to_host()
        np.testing.assert_allclose(st.concentrations(), g["y_solves"][i], rtol=RTOL, atol=ATOL)
