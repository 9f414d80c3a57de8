"""AlphaMinusJacobian and NormalizedError against micm's own known-answer
tests, on micm's 5-species test mechanism (GetSolver,
test/unit/solver/test_rosenbrock_solver_policy.hpp:1-60, state order kept):

* AlphaMinusJacobian (test_rosenbrock_solver_policy.hpp:62-115): a given
  Jacobian plus alpha = 42.042 on the diagonal, exactly;
* NormalizedError (test/unit/cuda/solver/test_cuda_rosenbrock.cpp:24-129):
  constant fills (1, 2, 3) and cell- and species-dependent fills with atol
  scaled by (1 + 0.01 i), against the formula
  max(sqrt(sum (e / (atol + rtol max(|y|, |ynew|)))^2 / (cells * species)), 1e-10)
  within micm's tolerances (1e-14 and 1e-11 relative), or the rounding bound
  of a sequential sum of cells * species terms where that is larger."""
import math

import numpy as np
import pytest

import oracle
from micm_b200.mechanism import Mechanism, arrhenius

# micm's instantiations use these cell counts (with several vector lengths)
CELLS = [1, 2, 7, 29, 37, 77, 219, 5599]


def get_solver_mechanism():
    m = Mechanism(species=["foo", "bar", "baz", "quz", "quuz"], reactions=[], name="get_solver", reorder_state=False)
    m.add(arrhenius(A=2.0e-11, B=0.0, C=110.0), [0, 2], [(1, 1.0), (4, 2.4)])
    m.add(arrhenius(A=1.0e-6), [1], [(0, 1.0), (3, 1.4)])
    m.add(arrhenius(A=3.5e-6), [3], [])
    return m


NEG_JAC = {(0, 0): lambda c: -12.2, (0, 1): lambda c: -24.3 * (c + 2), (0, 2): lambda c: -42.3,
           (1, 0): lambda c: -0.43, (1, 1): lambda c: -23.4, (1, 2): lambda c: -83.4 / (c + 3),
           (2, 0): lambda c: -4.74, (2, 2): lambda c: -6.91, (3, 1): lambda c: -59.1, (3, 3): lambda c: -83.4,
           (4, 0): lambda c: -78.5, (4, 2): lambda c: -53.6, (4, 4): lambda c: -1.0}


def fills(n, S, atol, rtol, kind):
    if kind == "const":
        y, yn, e = np.full((n, S), 1.0), np.full((n, S), 2.0), np.full((n, S), 3.0)
        atol = np.asarray(atol, dtype=np.float64)
    else:
        i = np.arange(n)[:, None].astype(np.float64)
        j = np.arange(S)[None, :].astype(np.float64)
        y = 7.7 * i + j
        yn = -13.9 / (j + 1) - i
        e = 81.57 / (i + 7) / (j + 3)
        atol = np.array([a * (1 + k * 0.01) for k, a in enumerate(atol)])
    return y, yn, e, atol


def expected_error(y, yn, e, atol, rtol, kind):
    total = 0.0
    rows = y[:1] if kind == "const" else y       # micm's constant case sums one cell, all cells are equal
    for c in range(len(rows)):
        for s in range(y.shape[1]):
            scale = atol[s] + rtol * max(abs(y[c, s]), abs(yn[c, s]))
            total += e[c, s] * e[c, s] / (scale * scale)
    count = y.shape[1] if kind == "const" else y.size
    return max(math.sqrt(total / count), 1.0e-10)


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("kind,tol", [("const", 1e-14), ("diff", 1e-11)])
@pytest.mark.parametrize("n", [1, 7, 219])
def test_micm_normalized_error_formula(kind, tol, n):
    mech = get_solver_mechanism()
    ref = oracle.Reference(mech, tableau=3)
    S = mech.n_species
    y, yn, e, atol = fills(n, S, mech.atol(), mech.relative_tolerance, kind)
    np.testing.assert_array_equal(ref.species_columns, np.arange(S))    # state order kept
    ref.atol_columns = atol
    got = ref.normalized_error(y, yn, e)
    want = expected_error(y, yn, e, atol, mech.relative_tolerance, kind)
    assert abs(got - want) <= tol * want


@pytest.mark.gpu
@pytest.mark.parametrize("L,n", [(1, 1), (2, 2), (7, 7), (29, 29), (37, 37), (77, 77), (1, 219), (128, 5599)])
def test_gpu_alpha_minus_jacobian(cuda_device, L, n):
    from micm_b200 import Solver
    from micm_b200 import solver as sv
    from micm_b200._native import check, lib
    from gpu_helpers import download_cols, upload_cols
    solver = Solver(get_solver_mechanism(), 3, vector_length=L)
    st = solver.get_state(n)
    rows, cols = solver.compiled.rows, solver.compiled.cols
    jac = np.zeros((n, len(rows)))
    for e, (r, c) in enumerate(zip(rows, cols)):
        if (r, c) in NEG_JAC:
            jac[:, e] = [NEG_JAC[(r, c)](i) for i in range(n)]
    upload_cols(st, sv.BUF_JACOBIAN, jac)
    check(lib().micmb_alpha_minus_jacobian(solver.handle, st.handle, 42.042))
    out = download_cols(st, sv.BUF_JACOBIAN, len(rows))
    want = jac.copy()
    for e, (r, c) in enumerate(zip(rows, cols)):
        if r == c:
            want[:, e] = 42.042 + jac[:, e]
    np.testing.assert_array_equal(out, want)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,tol", [("const", 1e-14), ("diff", 1e-11)])
@pytest.mark.parametrize("n", CELLS)
def test_gpu_normalized_error(cuda_device, kind, tol, n):
    from micm_b200 import Solver
    from micm_b200 import solver as sv
    from micm_b200._native import check, lib
    from gpu_helpers import upload_cols
    import ctypes
    mech = get_solver_mechanism()
    solver = Solver(mech, 3, vector_length=32)
    st = solver.get_state(n)
    S = mech.n_species
    y, yn, e, atol = fills(n, S, mech.atol(), mech.relative_tolerance, kind)
    upload_cols(st, sv.BUF_VARIABLES, y)
    upload_cols(st, sv.BUF_SCRATCH_Y, yn)
    upload_cols(st, sv.BUF_FORCING, e)
    st.upload(sv.BUF_ABSOLUTE_TOLERANCE, atol)
    out = ctypes.c_double(0.0)
    check(lib().micmb_normalized_error(solver.handle, st.handle, ctypes.byref(out), None))
    want = expected_error(y, yn, e, atol, mech.relative_tolerance, kind)
    # the global norm adds its n * S terms one after another, in micm's CPU
    # order (so it equals micm's CPU solver bit for bit); that rounding grows
    # with the count, up to about n * S * 2.2e-16 relative (micm's own 1e-14
    # is set for its CUDA tree reduction)
    tol = max(tol, n * S * 2.2e-16)
    assert abs(out.value - want) <= tol * want, (out.value, want)
