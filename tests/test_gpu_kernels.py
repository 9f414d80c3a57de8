"""Per-kernel parity on the GPU against micm's own CPU functions on the same
inputs (micm's CUDA unit tests compare the same stages:
test/unit/cuda/process/test_cuda_process_set.cpp, test_cuda_lu_decomposition_mozart_in_place.cpp,
test_cuda_linear_solver_in_place.cpp, test/unit/cuda/solver/test_cuda_rosenbrock.cpp)."""
import numpy as np
import pytest

import oracle
from micm_b200 import Solver, synthetic
from micm_b200 import solver as sv

from gpu_helpers import download_cols, make_state, upload_cols
from mechanisms import all_rate_types, all_rate_types_inputs

pytestmark = pytest.mark.gpu


def _case(name, n, seed):
    if name == "all_kinds":
        return all_rate_types(), all_rate_types_inputs(n, seed)
    m = synthetic.synthetic_mechanism(210, 440, seed=2101) if name == "syn210" else \
        synthetic.synthetic_mechanism(60, 120, seed=601)
    return m, synthetic.cell_inputs(m, n, seed)


@pytest.mark.parametrize("name,L", [("all_kinds", 1), ("all_kinds", 32), ("syn60", 3), ("syn210", 128)])
def test_rate_constants(cuda_device, name, L):
    m, inp = _case(name, 77, 3)
    ref = oracle.Reference(m)
    k_ref = ref.rate_constants(inp["temperature"], inp["pressure"], inp["air_density"], inp["custom_params"])
    solver = Solver(m, 3, vector_length=L)
    st = make_state(solver, inp)
    solver.update_state_parameters(st)
    k = st.rate_constants()
    np.testing.assert_allclose(k, k_ref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("name,L", [("all_kinds", 4), ("syn210", 32)])
def test_forcing_and_jacobian(cuda_device, name, L):
    m, inp = _case(name, 65, 4)
    ref = oracle.Reference(m)
    solver = Solver(m, 3, vector_length=L)
    st = make_state(solver, inp)
    rng = np.random.default_rng(9)
    k = rng.lognormal(-2, 4, size=(65, m.n_reactions))
    y = ref.y_to_columns(inp["concentrations"])
    upload_cols(st, sv.BUF_RATE_CONSTANTS, k)
    upload_cols(st, sv.BUF_VARIABLES, y)
    upload_cols(st, sv.BUF_FORCING, np.zeros((65, m.n_species)))
    st_check = 0
    from micm_b200._native import check, lib
    check(lib().micmb_add_forcing_terms(solver.handle, st.handle))
    f = download_cols(st, sv.BUF_FORCING, m.n_species)
    f_ref = ref.forcing(k, y)
    np.testing.assert_array_equal(f, f_ref)  # same operations, same order, separate rounding
    nnz = solver.compiled.info["jacobian_nnz"]
    upload_cols(st, sv.BUF_JACOBIAN, np.zeros((65, nnz)))
    check(lib().micmb_subtract_jacobian_terms(solver.handle, st.handle))
    j = download_cols(st, sv.BUF_JACOBIAN, nnz)
    j_ref = ref.jacobian(k, y)
    np.testing.assert_array_equal(j, j_ref)
    check(lib().micmb_alpha_minus_jacobian(solver.handle, st.handle, 12.5))
    ja = download_cols(st, sv.BUF_JACOBIAN, nnz)
    diag = ref.rows == ref.cols
    expect = j_ref.copy()
    expect[:, diag] += 12.5
    np.testing.assert_array_equal(ja, expect)


@pytest.mark.parametrize("name,L", [("syn60", 1), ("syn210", 32), ("syn210", 77)])
def test_lu_and_linear_solve(cuda_device, name, L):
    m, inp = _case(name, 70, 5)
    ref = oracle.Reference(m)
    solver = Solver(m, 3, vector_length=L)
    st = make_state(solver, inp)
    rng = np.random.default_rng(11)
    nnz = ref.nnz
    a = rng.normal(size=(70, nnz))
    diag = ref.rows == ref.cols
    a[:, diag] += 50.0 + np.abs(a[:, diag])
    upload_cols(st, sv.BUF_JACOBIAN, a)
    from micm_b200._native import check, lib
    check(lib().micmb_lu_decompose(solver.handle, st.handle))
    lu = download_cols(st, sv.BUF_JACOBIAN, nnz)
    lu_ref = ref.decompose(a)
    # same operations in the same order with separate rounding: bit-for-bit
    np.testing.assert_array_equal(lu, lu_ref)
    b = rng.normal(size=(70, m.n_species))
    upload_cols(st, sv.BUF_FORCING, b)
    check(lib().micmb_linear_solve(solver.handle, st.handle))
    x = download_cols(st, sv.BUF_FORCING, m.n_species)
    x_ref = ref.linear_solve(lu_ref, b)
    np.testing.assert_array_equal(x, x_ref)


def test_normalized_error(cuda_device):
    m, inp = _case("syn210", 300, 6)
    ref = oracle.Reference(m)
    solver = Solver(m, 3, vector_length=64)
    st = make_state(solver, inp)
    rng = np.random.default_rng(12)
    y = 10 ** rng.uniform(-14, -6, size=(300, m.n_species))
    ynew = y * (1 + 1e-5 * rng.normal(size=y.shape))
    err = 1e-9 * rng.normal(size=y.shape)
    upload_cols(st, sv.BUF_VARIABLES, y)
    upload_cols(st, sv.BUF_SCRATCH_Y, ynew)
    upload_cols(st, sv.BUF_FORCING, err)
    import ctypes as C
    from micm_b200._native import check, lib
    g = C.c_double()
    per = np.zeros(300)
    check(lib().micmb_normalized_error(solver.handle, st.handle, C.byref(g), per.ctypes.data_as(C.POINTER(C.c_double))))
    e_ref = ref.normalized_error(y, ynew, err)
    assert abs(g.value - e_ref) <= 1e-12 * e_ref
    for c in (0, 17, 299):
        e1 = ref.normalized_error(y[c:c + 1], ynew[c:c + 1], err[c:c + 1])
        assert abs(per[c] - e1) <= 1e-12 * e1
