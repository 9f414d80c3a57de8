"""micmb_normalized_error_noalloc against micmb_normalized_error: two calls in
a row on changing inputs give the same bits, and states beyond the fixed
scratch are refused.  Collected last (file name), and self-contained so it
passes alone as well."""
import ctypes as C

import numpy as np
import pytest

from micm_b200 import Solver, synthetic
from micm_b200 import solver as sv
from micm_b200._native import check, lib
from micm_b200.mechanism import to_vector_layout

pytestmark = pytest.mark.gpu


def _norms(solver, st):
    ref = C.c_double(0.0)
    check(lib().micmb_normalized_error(solver.handle, st.handle, C.byref(ref), None))
    out = C.c_double(-1.0)
    check(lib().micmb_normalized_error_noalloc(solver.handle, st.handle, C.byref(out)))
    return ref.value, out.value


def test_noalloc_matches_allocating_entry_point(cuda_device):
    mech = synthetic.synthetic_mechanism(210, 440, seed=2101)
    n, L = 1000, 32
    solver = Solver(mech, 4, vector_length=L)
    st = solver.get_state(n)
    st.set_inputs(synthetic.cell_inputs(mech, n, 31))
    st.sync_inputs_to_device()
    rng = np.random.default_rng(8)
    y = st.variables
    for call in range(2):
        ynew = y * (1.0 + 1e-3 * rng.normal(size=y.shape))
        err = 1e-4 * y * rng.normal(size=y.shape) * (call + 1)
        st.upload(sv.BUF_SCRATCH_Y, to_vector_layout(ynew, L))
        st.upload(sv.BUF_FORCING, to_vector_layout(err, L))
        ref, out = _norms(solver, st)
        assert out == ref and out > 0.0


def test_noalloc_refuses_more_cells_than_its_scratch(cuda_device):
    mech = synthetic.readme_mechanism()
    solver = Solver(mech, 3, vector_length=1)
    st = solver.get_state(65537)
    out = C.c_double(-1.0)
    rc = lib().micmb_normalized_error_noalloc(solver.handle, st.handle, C.byref(out))
    assert rc == -1 and out.value == -1.0
    assert b"65536" in lib().micmb_last_error()
