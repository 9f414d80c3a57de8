"""ctypes mirror of the plain-C structs of include/micmb.h."""
from __future__ import annotations

import ctypes as C
from typing import Dict

import numpy as np

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)


class MechanismDesc(C.Structure):
    _fields_ = [
        ("n_species", C.c_int32),
        ("n_reactions", C.c_int32),
        ("rate_type", i32p),
        ("rate_params", f64p),
        ("reactant_start", i32p),
        ("reactant_species", i32p),
        ("product_start", i32p),
        ("product_species", i32p),
        ("product_yield", f64p),
        ("n_parameterized", C.c_int32),
        ("parameterized_coef", f64p),
        ("reorder_state", C.c_int32),
        ("n_constraints", C.c_int32),
        ("constraint_type", i32p),
        ("constraint_species", i32p),
        ("constraint_term_start", i32p),
        ("constraint_term_species", i32p),
        ("constraint_term_coef", f64p),
        ("constraint_n_reactants", i32p),
        ("constraint_params", f64p),
    ]


class RosenbrockParams(C.Structure):
    _fields_ = [
        ("stages", C.c_int32),
        ("max_number_of_steps", C.c_int32),
        ("round_off", C.c_double),
        ("factor_min", C.c_double),
        ("factor_max", C.c_double),
        ("rejection_factor_decrease", C.c_double),
        ("safety_factor", C.c_double),
        ("h_min", C.c_double),
        ("h_max", C.c_double),
        ("h_start", C.c_double),
        ("new_function_evaluation", C.c_int32 * 6),
        ("estimator_of_local_order", C.c_double),
        ("a", C.c_double * 15),
        ("c", C.c_double * 15),
        ("m", C.c_double * 6),
        ("e", C.c_double * 6),
        ("alpha", C.c_double * 6),
        ("gamma", C.c_double * 6),
        ("constraint_init_max_iterations", C.c_int32),
        ("constraint_init_tolerance", C.c_double),
    ]


class SolverStats(C.Structure):
    _fields_ = [
        ("function_calls", C.c_int64),
        ("jacobian_updates", C.c_int64),
        ("number_of_steps", C.c_int64),
        ("accepted", C.c_int64),
        ("rejected", C.c_int64),
        ("decompositions", C.c_int64),
        ("solves", C.c_int64),
        ("final_time", C.c_double),
        ("state", C.c_int32),
        ("cells_not_converged", C.c_int32),
        ("constraint_init_iterations", C.c_int64),
    ]

    def as_dict(self) -> Dict[str, float]:
        return {name: getattr(self, name) for name, _ in self._fields_}


class MechanismInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "n_species", "n_reactions", "n_custom_params", "jacobian_nnz", "jacobian_nnz_unfilled",
        "lu_updates", "lu_lower", "n_jacobian_terms", "n_forcing_terms", "n_jacobian_infos",
        "lu_levels", "forward_levels", "backward_levels", "blocked_schedules", "lu_blocked_ops")]

    def as_dict(self) -> Dict[str, int]:
        return {name: getattr(self, name) for name, _ in self._fields_}


class FusedConfig(C.Structure):
    _fields_ = [("cells_per_cta", C.c_int32), ("lu_in_shared", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("ring_slots", C.c_int32), ("variant", C.c_int32)]


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class DescHolder:
    """Owns the numpy arrays behind a MechanismDesc."""

    def __init__(self, flat: Dict[str, np.ndarray]):
        self.arrays = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v)
                       for k, v in flat.items()}
        a = self.arrays
        self.desc = MechanismDesc(
            n_species=int(a["n_species"]),
            n_reactions=int(a["n_reactions"]),
            rate_type=ptr(a["rate_type"], C.c_int32),
            rate_params=ptr(a["rate_params"], C.c_double),
            reactant_start=ptr(a["reactant_start"], C.c_int32),
            reactant_species=ptr(_nonempty(a, "reactant_species", np.int32), C.c_int32),
            product_start=ptr(a["product_start"], C.c_int32),
            product_species=ptr(_nonempty(a, "product_species", np.int32), C.c_int32),
            product_yield=ptr(_nonempty(a, "product_yield", np.float64), C.c_double),
            n_parameterized=int(a["n_parameterized"]),
            parameterized_coef=ptr(a["parameterized_coef"], C.c_double),
            reorder_state=int(a["reorder_state"]),
            n_constraints=int(a.get("n_constraints", 0)),
        )
        if self.desc.n_constraints:
            d = self.desc
            d.constraint_type = ptr(a["constraint_type"], C.c_int32)
            d.constraint_species = ptr(a["constraint_species"], C.c_int32)
            d.constraint_term_start = ptr(a["constraint_term_start"], C.c_int32)
            d.constraint_term_species = ptr(_nonempty(a, "constraint_term_species", np.int32), C.c_int32)
            d.constraint_term_coef = ptr(_nonempty(a, "constraint_term_coef", np.float64), C.c_double)
            d.constraint_n_reactants = ptr(a["constraint_n_reactants"], C.c_int32)
            d.constraint_params = ptr(a["constraint_params"], C.c_double)


def _nonempty(a, key, dtype):
    if a[key].size == 0:
        a[key] = np.zeros(1, dtype=dtype)
    return a[key]


class BackwardEulerParams(C.Structure):
    """micm::BackwardEulerSolverParameters (backward_euler_solver_parameters.hpp:17-29)."""
    _fields_ = [
        ("small", C.c_double),
        ("h_start", C.c_double),
        ("max_number_of_steps", C.c_int32),
        ("n_time_step_reductions", C.c_int32),
        ("time_step_reductions", C.c_double * 8),
    ]
