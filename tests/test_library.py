"""The C-ABI library loads and exports every entry point include/micmb.h declares;
the host-side compile works without a GPU; the product refuses to run without one."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "micmb.h")).read()
    return sorted(set(re.findall(r"\b(micmb_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    from micm_b200 import _native
    lib = ctypes.CDLL(_native.LIB_PATH)
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_checkers_load():
    import oracle
    assert oracle.reference_available() and oracle.restatement_available()
    ctypes.CDLL(oracle.REF_LIB)
    ctypes.CDLL(oracle.ORACLE_LIB)


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from micm_b200 import Solver, synthetic
    from micm_b200._native import MicmbError
    with pytest.raises(MicmbError) as e:
        Solver(synthetic.readme_mechanism(), 3)
    assert e.value.code == -6  # MICMB_ERR_NO_DEVICE


def test_tableaus_match_reference_values():
    """The published tableaus the library returns are micm's
    (rosenbrock_solver_parameters.hpp:152-434); spot-check stage counts and a few entries."""
    from micm_b200.solver import RosenbrockSolverParameters as P
    p3 = P.three_stage()
    assert p3.stages == 3 and p3.gamma[0] == 0.43586652150845899941601945119356
    p4 = P.four_stage()
    assert p4.stages == 4 and list(p4.new_function_evaluation)[:4] == [1, 1, 1, 0]
    assert p4.m[3] == 0.1093502252409163E+01 and p4.e[3] == -0.1093502252409163E+01
    p6 = P.six_stage_differential_algebraic()
    assert p6.stages == 6 and p6.c[14] == -0.6058818238834054E+01 and p6.a[14] == 1.0
    assert P.two_stage().gamma[0] == 1.0 + 1.0 / np.sqrt(2.0)
