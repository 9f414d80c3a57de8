"""TEST INFRASTRUCTURE: checkers for the B200 solver.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this package;
the product never does.

Two checkers live here:

* :class:`Reference` -- micm itself (oracle/_ref/libmicm_ref.so, built from the
  reference's own headers by oracle/Makefile through ref_bridge.cpp).
* :class:`Restatement` -- oracle.c, a plain-C restatement of micm's Rosenbrock
  path plus the discrete adjoint micm does not have (oracle/liboracle.so).

Arrays at these interfaces are row-major [cell][column] in state columns
(species after Markowitz reordering, reactions after the type sort).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

from micm_b200._abi import DescHolder
from micm_b200.mechanism import Mechanism

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libmicm_ref.so")
# micm built for speed (FMA contraction, AVX2): the CPU baseline, not a parity checker
REF_LIB_FAST = os.path.join(HERE, "_ref", "libmicm_ref_fast.so")
ORACLE_LIB = os.path.join(HERE, "liboracle.so")

_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)

STATS_FIELDS = ("function_calls", "jacobian_updates", "number_of_steps", "accepted", "rejected",
                "decompositions", "solves", "state")


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


_ref = {}


def reference_available(fast: bool = False) -> bool:
    return os.path.exists(REF_LIB_FAST if fast else REF_LIB)


def _load_ref(fast: bool = False):
    if fast not in _ref:
        lib = C.CDLL(REF_LIB_FAST if fast else REF_LIB)
        lib.mref_last_error.restype = C.c_char_p
        lib.mref_create.restype = C.c_void_p
        lib.mref_create.argtypes = [C.c_void_p, _f64p, C.c_double, C.c_int]
        lib.mref_destroy.argtypes = [C.c_void_p]
        for name in ("mref_species_columns", "mref_reaction_columns", "mref_custom_param_columns"):
            getattr(lib, name).argtypes = [C.c_void_p, _i32p]
        lib.mref_n_custom_params.argtypes = [C.c_void_p]
        lib.mref_jacobian_pattern.argtypes = [C.c_void_p, _i32p, _i32p]
        lib.mref_rate_constants.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p, _f64p, _f64p]
        lib.mref_forcing.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p]
        lib.mref_jacobian.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p]
        lib.mref_decompose.argtypes = [C.c_void_p, C.c_int, _f64p]
        lib.mref_linear_solve.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p]
        lib.mref_normalized_error.restype = C.c_double
        lib.mref_normalized_error.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p, _f64p, C.c_double]
        lib.mref_solve_global.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, _f64p, _f64p, _f64p,
                                          _f64p, _f64p, _i64p]
        lib.mref_solve_per_cell.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, _f64p, _f64p, _f64p,
                                            _f64p, _f64p, _i64p, C.c_int]
        if hasattr(lib, "mref_backward_euler_global"):
            lib.mref_backward_euler_global.argtypes = [C.c_void_p, C.c_int, C.c_double, _f64p, _f64p, _f64p,
                                                       _f64p, _f64p, _i64p]
        if hasattr(lib, "mref_backward_euler_per_cell"):
            lib.mref_backward_euler_per_cell.argtypes = [C.c_void_p, C.c_int, C.c_double, _f64p, _f64p, _f64p,
                                                         _f64p, _f64p, _i64p]
        if hasattr(lib, "mref_solve_groups_v128"):
            lib.mref_solve_groups_v128.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, _f64p, _f64p,
                                                   _f64p, _f64p, _f64p, _i64p, C.c_int]
        _ref[fast] = lib
    return _ref[fast]


def _stats_rows(raw: np.ndarray):
    out = []
    for row in raw:
        d = {k: int(row[i]) for i, k in enumerate(STATS_FIELDS)}
        d["final_time"] = float(row[8:9].view(np.float64)[0])
        d["constraint_init_iterations"] = int(row[9])
        out.append(d)
    return out


class Reference:
    """micm's own CPU Rosenbrock (in-place Mozart LU, vector ordering).
    fast=True loads the build for speed (the CPU baseline) instead of the
    bit-exact parity build."""

    def __init__(self, mech: Mechanism, tableau: int = 3, fast: bool = False):
        self.lib = _load_ref(fast)
        self.mech = mech
        self._desc = DescHolder(mech.flat())
        atol = np.ascontiguousarray(mech.atol())
        self.handle = self.lib.mref_create(C.byref(self._desc.desc), _p(atol), mech.relative_tolerance,
                                           int(tableau))
        if not self.handle:
            raise RuntimeError("mref_create: " + self.lib.mref_last_error().decode())
        S, R = mech.n_species, mech.n_reactions
        self.S, self.R = S, R
        self.species_columns = np.zeros(S, np.int32)
        self.lib.mref_species_columns(self.handle, _p(self.species_columns, C.c_int32))
        self.reaction_columns = np.zeros(R, np.int32)
        self.lib.mref_reaction_columns(self.handle, _p(self.reaction_columns, C.c_int32))
        self.param_columns = np.zeros(R, np.int32)
        self.lib.mref_custom_param_columns(self.handle, _p(self.param_columns, C.c_int32))
        self.n_params = self.lib.mref_n_custom_params(self.handle)
        nnz = self.lib.mref_jacobian_pattern(self.handle, None, None)
        self.rows = np.zeros(nnz, np.int32)
        self.cols = np.zeros(nnz, np.int32)
        self.lib.mref_jacobian_pattern(self.handle, _p(self.rows, C.c_int32), _p(self.cols, C.c_int32))
        self.nnz = nnz
        self.atol_columns = np.zeros(S)
        self.atol_columns[self.species_columns] = atol

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.mref_destroy(self.handle)
            self.handle = None

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.mref_last_error().decode())

    # system order -> state columns
    def y_to_columns(self, y_sys: np.ndarray) -> np.ndarray:
        out = np.zeros_like(y_sys)
        out[:, self.species_columns] = y_sys
        return np.ascontiguousarray(out)

    def y_from_columns(self, y_cols: np.ndarray) -> np.ndarray:
        return np.ascontiguousarray(y_cols[:, self.species_columns])

    def params_to_columns(self, params_labels: np.ndarray) -> np.ndarray:
        """custom params in label order (Mechanism.custom_param_labels) -> micm columns.
        Label order and micm's column order coincide by construction; kept explicit."""
        return np.ascontiguousarray(params_labels.reshape(len(params_labels), -1))

    def rate_constants(self, T, P, rho, params):
        n = len(T)
        k = np.zeros((n, self.R))
        params = np.ascontiguousarray(params if params.size else np.zeros((n, 1)))
        self._check(self.lib.mref_rate_constants(self.handle, n, _p(np.ascontiguousarray(T)),
                                                 _p(np.ascontiguousarray(P)), _p(np.ascontiguousarray(rho)),
                                                 _p(params), _p(k)))
        return k

    def forcing(self, k, y_cols):
        n = len(k)
        f = np.zeros((n, self.S))
        self._check(self.lib.mref_forcing(self.handle, n, _p(np.ascontiguousarray(k)),
                                          _p(np.ascontiguousarray(y_cols)), _p(f)))
        return f

    def jacobian(self, k, y_cols):
        n = len(k)
        j = np.zeros((n, self.nnz))
        self._check(self.lib.mref_jacobian(self.handle, n, _p(np.ascontiguousarray(k)),
                                           _p(np.ascontiguousarray(y_cols)), _p(j)))
        return j

    def decompose(self, a):
        lu = np.ascontiguousarray(a, dtype=np.float64).copy()
        self._check(self.lib.mref_decompose(self.handle, len(lu), _p(lu)))
        return lu

    def linear_solve(self, lu, b):
        x = np.ascontiguousarray(b, dtype=np.float64).copy()
        self._check(self.lib.mref_linear_solve(self.handle, len(x), _p(np.ascontiguousarray(lu)), _p(x)))
        return x

    def normalized_error(self, y, ynew, err, rtol=None):
        rtol = self.mech.relative_tolerance if rtol is None else rtol
        return self.lib.mref_normalized_error(self.handle, len(y), _p(np.ascontiguousarray(y)),
                                              _p(np.ascontiguousarray(ynew)), _p(np.ascontiguousarray(err)),
                                              _p(self.atol_columns), float(rtol))

    def solve_global(self, inputs: Dict[str, np.ndarray], dt: float, n_solves: int = 1):
        """One multi-cell State, micm's single step size for all cells."""
        y = self.y_to_columns(inputs["concentrations"])
        n = len(y)
        stats = np.zeros((n_solves, 10), np.int64)
        params = np.ascontiguousarray(inputs["custom_params"] if inputs["custom_params"].size
                                      else np.zeros((n, 1)))
        self._check(self.lib.mref_solve_global(
            self.handle, n, float(dt), int(n_solves), _p(inputs["temperature"]), _p(inputs["pressure"]),
            _p(inputs["air_density"]), _p(params), _p(y), _p(stats, C.c_int64)))
        return self.y_from_columns(y), _stats_rows(stats)

    def solve_groups_v128(self, inputs: Dict[str, np.ndarray], dt: float, group: int = 1024, n_solves: int = 1,
                          threads: int = 0):
        """micm with vector ordering L = 128: one State (one step size) per group
        of `group` cells, groups over host threads.  Returns (y_final [n,S]
        system order, stats rows per group)."""
        if not hasattr(self.lib, "mref_solve_groups_v128"):
            raise RuntimeError("oracle/_ref/libmicm_ref.so predates mref_solve_groups_v128; rebuild it")
        y = self.y_to_columns(inputs["concentrations"])
        n = len(y)
        stats = np.zeros((max(-(-n // group), 1), 10), np.int64)
        params = np.ascontiguousarray(inputs["custom_params"] if inputs["custom_params"].size
                                      else np.zeros((n, 1)))
        threads = threads or (os.cpu_count() or 1)
        self._check(self.lib.mref_solve_groups_v128(
            self.handle, n, int(group), float(dt), int(n_solves), _p(inputs["temperature"]),
            _p(inputs["pressure"]), _p(inputs["air_density"]), _p(params), _p(y), _p(stats, C.c_int64),
            int(threads)))
        return self.y_from_columns(y), stats

    def backward_euler_per_cell(self, inputs: Dict[str, np.ndarray], dt: float):
        """micm's Backward Euler, a 1-cell State per cell, one Solve(dt) each:
        (y_final [n,S] system order, stats rows per cell)."""
        if not hasattr(self.lib, "mref_backward_euler_per_cell"):
            raise RuntimeError("oracle/_ref/libmicm_ref.so predates mref_backward_euler_per_cell; rebuild it")
        y = self.y_to_columns(inputs["concentrations"])
        n = len(y)
        stats = np.zeros((n, 10), np.int64)
        params = np.ascontiguousarray(inputs["custom_params"] if inputs["custom_params"].size
                                      else np.zeros((n, 1)))
        self._check(self.lib.mref_backward_euler_per_cell(
            self.handle, n, float(dt), _p(inputs["temperature"]), _p(inputs["pressure"]),
            _p(inputs["air_density"]), _p(params), _p(y), _p(stats, C.c_int64)))
        return self.y_from_columns(y), stats

    def backward_euler_global(self, inputs: Dict[str, np.ndarray], dt: float):
        """micm's Backward Euler on one n-cell State, one Solve(dt):
        (y_final [n,S] system order, stats row [10])."""
        if not hasattr(self.lib, "mref_backward_euler_global"):
            raise RuntimeError("oracle/_ref/libmicm_ref.so predates mref_backward_euler_global; rebuild it")
        y = self.y_to_columns(inputs["concentrations"])
        n = len(y)
        stats = np.zeros(10, np.int64)
        params = np.ascontiguousarray(inputs["custom_params"] if inputs["custom_params"].size
                                      else np.zeros((n, 1)))
        self._check(self.lib.mref_backward_euler_global(
            self.handle, n, float(dt), _p(inputs["temperature"]), _p(inputs["pressure"]),
            _p(inputs["air_density"]), _p(params), _p(y), _p(stats, C.c_int64)))
        return self.y_from_columns(y), stats

    def solve_per_cell(self, inputs: Dict[str, np.ndarray], dt: float, n_solves: int = 1,
                       threads: int = 0):
        """A 1-cell State per cell; returns (y_final [n,S] system order, stats rows per cell)."""
        y = self.y_to_columns(inputs["concentrations"])
        n = len(y)
        stats = np.zeros((n, 10), np.int64)
        params = np.ascontiguousarray(inputs["custom_params"] if inputs["custom_params"].size
                                      else np.zeros((n, 1)))
        threads = threads or (os.cpu_count() or 1)
        self._check(self.lib.mref_solve_per_cell(
            self.handle, n, float(dt), int(n_solves), _p(inputs["temperature"]), _p(inputs["pressure"]),
            _p(inputs["air_density"]), _p(params), _p(y), _p(stats, C.c_int64), int(threads)))
        return self.y_from_columns(y), stats


_om = None


# double exchange(double value, int op, void* user): op EXCHANGE_SUM, the job's sum
# of the shards' error sums in rank order; op EXCHANGE_MAX, the job's combination
# of the shards' encoded maxima (max_combine)
EXCHANGE_FN = C.CFUNCTYPE(C.c_double, C.c_double, C.c_int, C.c_void_p)
EXCHANGE_SUM, EXCHANGE_MAX = 0, 1


def max_combine(values):
    """The shards' encoded maxima of the constraint initialisation combined in
    rank order: NaN when any is NaN, +Inf when any is infinite, else the largest
    (oracle.c om_max_combine)."""
    out = 0.0
    for v in values:
        v = float(v)
        if np.isnan(out) or np.isnan(v):
            out = float("nan")
        elif np.isinf(out) or np.isinf(v):
            out = float("inf")
        else:
            out = max(out, v)
    return out


def _load_oracle():
    global _om
    if _om is None:
        lib = C.CDLL(ORACLE_LIB)
        lib.om_create.restype = C.c_void_p
        lib.om_create.argtypes = [C.c_void_p]
        lib.om_destroy.argtypes = [C.c_void_p]
        lib.om_last_error.restype = C.c_char_p
        lib.om_n_params.argtypes = [C.c_void_p]
        lib.om_nnz.argtypes = [C.c_void_p]
        lib.om_species_columns.argtypes = [C.c_void_p, _i32p]
        lib.om_reaction_columns.argtypes = [C.c_void_p, _i32p]
        lib.om_jacobian_pattern.argtypes = [C.c_void_p, _i32p, _i32p]
        lib.om_rate_constants.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p, _f64p, _f64p]
        lib.om_solve_per_cell.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, _f64p, _f64p, C.c_double,
                                          _f64p, _i64p, C.c_int]
        lib.om_adjoint_per_cell.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, _f64p, _f64p,
                                            C.c_double, _f64p, _f64p, _f64p, _f64p, _f64p, C.c_int, C.c_int]
        lib.om_replay_per_cell.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _f64p, _f64p, _i32p, C.c_int, _f64p]
        lib.om_solve_global.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, _f64p, _f64p, _f64p,
                                        C.c_double, _f64p, _i64p, C.c_int, _i32p, EXCHANGE_FN, C.c_void_p, C.c_int64]
        lib.om_n_eq.argtypes = [C.c_void_p]
        lib.om_constraint_params.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p]
        lib.om_constraint_params.restype = None
        lib.om_solve_per_cell_keq.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, _f64p, _f64p, _f64p,
                                              C.c_double, _f64p, _i64p, C.c_int]
        lib.om_set_correctly_rounded.argtypes = [C.c_void_p, C.c_int]
        lib.om_set_correctly_rounded.restype = None
        lib.om_math_eval.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p, C.c_int64]
        lib.om_math_eval.restype = None
        lib.om_backward_euler_global.argtypes = [C.c_void_p, C.c_int, C.c_double, _f64p, _f64p, C.c_double,
                                                 _f64p, _i64p]
        lib.om_backward_euler_per_cell.argtypes = [C.c_void_p, C.c_int, C.c_double, _f64p, _f64p, C.c_double,
                                                   _f64p, _i64p]
        lib.om_step_sizes_per_cell.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, _f64p, _f64p,
                                               C.c_double, _f64p, C.c_int, _f64p, _i32p]
        _om = lib
    return _om


def restatement_available() -> bool:
    return os.path.exists(ORACLE_LIB)


def tableau(kind: int):
    """micm's tableau in micmb_rosenbrock_params form, restated from
    rosenbrock_solver_parameters.hpp:152-434 through the reference bridge-free
    path: the values are the published coefficients (tests check they equal
    the library's own defaults)."""
    from micm_b200.solver import RosenbrockSolverParameters
    return RosenbrockSolverParameters.from_stages(kind)


class Restatement:
    """oracle.c: plain-C restatement of micm's Rosenbrock path + discrete adjoint."""

    def __init__(self, mech: Mechanism, tableau_kind: int = 3, params=None, correctly_rounded: bool = False):
        """correctly_rounded: exp, pow and log10 of the rate constants and the
        step-size factor correctly rounded (quad precision) instead of the C
        library's (micm's)."""
        self.lib = _load_oracle()
        self.mech = mech
        self._desc = DescHolder(mech.flat())
        self.handle = self.lib.om_create(C.byref(self._desc.desc))
        if not self.handle:
            raise RuntimeError("om_create: " + self.lib.om_last_error().decode())
        self.lib.om_set_correctly_rounded(self.handle, 1 if correctly_rounded else 0)
        self.S, self.R = mech.n_species, mech.n_reactions
        self.params = params if params is not None else tableau(tableau_kind)
        self.species_columns = np.zeros(self.S, np.int32)
        self.lib.om_species_columns(self.handle, _p(self.species_columns, C.c_int32))
        self.reaction_columns = np.zeros(max(self.R, 1), np.int32)
        self.lib.om_reaction_columns(self.handle, _p(self.reaction_columns, C.c_int32))
        self.reaction_columns = self.reaction_columns[: self.R]
        self.nnz = self.lib.om_nnz(self.handle)
        self.n_params = self.lib.om_n_params(self.handle)
        self.rows = np.zeros(self.nnz, np.int32)
        self.cols = np.zeros(self.nnz, np.int32)
        self.lib.om_jacobian_pattern(self.handle, _p(self.rows, C.c_int32), _p(self.cols, C.c_int32))
        self.atol_columns = np.zeros(self.S)
        self.atol_columns[self.species_columns] = mech.atol()

    def math_eval(self, fn: int, x, y=None):
        """exp (0), log10 (1) or pow (2) element-wise in this handle's mode."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(x if y is None else y, dtype=np.float64)
        out = np.empty_like(x)
        self.lib.om_math_eval(self.handle, int(fn), _p(x), _p(y), _p(out), len(x))
        return out

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.om_destroy(self.handle)
            self.handle = None

    def rate_constants(self, T, P, rho, params):
        n = len(T)
        k = np.zeros((n, max(self.R, 1)))
        params = np.ascontiguousarray(params if params.size else np.zeros((n, 1)))
        self.lib.om_rate_constants(self.handle, n, _p(np.ascontiguousarray(T)), _p(np.ascontiguousarray(P)),
                                   _p(np.ascontiguousarray(rho)), _p(params), _p(k))
        return k[:, : self.R]

    def _k(self, inputs):
        return np.ascontiguousarray(self.rate_constants(inputs["temperature"], inputs["pressure"],
                                                        inputs["air_density"], inputs["custom_params"]))

    def keq(self, temperature) -> np.ndarray:
        """K_eq(T) of every equilibrium constraint per cell [n, n_eq] (this handle's exp)."""
        T = np.ascontiguousarray(temperature, dtype=np.float64)
        out = np.zeros((len(T), max(self.lib.om_n_eq(self.handle), 1)))
        self.lib.om_constraint_params(self.handle, len(T), _p(T), _p(out))
        return out

    def solve_per_cell(self, inputs, dt, threads=0, k=None):
        """Per-cell step control; with constraints, micm's DAE Rosenbrock
        (stats[:, 9] = constraint-initialisation iterations)."""
        y = np.zeros_like(inputs["concentrations"])
        y[:, self.species_columns] = inputs["concentrations"]
        n = len(y)
        k = self._k(inputs) if k is None else np.ascontiguousarray(k)
        keq = self.keq(inputs["temperature"])
        stats = np.zeros((n, 10), np.int64)
        rc = self.lib.om_solve_per_cell_keq(self.handle, C.byref(self.params), n, float(dt), _p(k), _p(keq),
                                            _p(self.atol_columns), self.mech.relative_tolerance, _p(y),
                                            _p(stats, C.c_int64), int(threads or os.cpu_count() or 1))
        if rc:
            raise RuntimeError(self.lib.om_last_error().decode())
        return np.ascontiguousarray(y[:, self.species_columns]), stats

    def backward_euler_per_cell(self, inputs, dt, k=None):
        """Backward Euler (micm's algorithm and default parameters), a 1-cell
        solve per cell: (y_final [n,S] system order, stats [n,10])."""
        y = np.zeros_like(inputs["concentrations"])
        y[:, self.species_columns] = inputs["concentrations"]
        y = np.ascontiguousarray(y)
        n = len(y)
        k = self._k(inputs) if k is None else np.ascontiguousarray(k)
        stats = np.zeros((n, 10), np.int64)
        rc = self.lib.om_backward_euler_per_cell(self.handle, n, float(dt), _p(k), _p(self.atol_columns),
                                                 self.mech.relative_tolerance, _p(y), _p(stats, C.c_int64))
        if rc:
            raise RuntimeError(self.lib.om_last_error().decode())
        return np.ascontiguousarray(y[:, self.species_columns]), stats

    def solve_global(self, inputs, dt, k=None, shards=None, exchange=None, total_cells=0):
        """Global step control (one step size for all cells), the error sum in
        the fixed order a GPU reproduces; with constraints, micm's DAE
        Rosenbrock on an n-cell State (one initialisation for all cells).
        shards: cell counts of consecutive shards (default one);
        exchange(value, op) makes the cells this rank's shard of a job over
        total_cells: op EXCHANGE_SUM returns the job's sum of the shard sums in
        rank order, op EXCHANGE_MAX the max_combine of the ranks' values.
        (y_final [n,S] system order, stats [10])."""
        y = np.zeros_like(inputs["concentrations"])
        y[:, self.species_columns] = inputs["concentrations"]
        y = np.ascontiguousarray(y)
        n = len(y)
        k = self._k(inputs) if k is None else np.ascontiguousarray(k)
        stats = np.zeros(10, np.int64)
        sizes = [n] if shards is None else list(shards)
        assert sum(sizes) == n
        starts = np.ascontiguousarray(np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32))
        keq = self.keq(inputs["temperature"])
        cb = EXCHANGE_FN(lambda v, op, _u: float(exchange(v, op))) if exchange else EXCHANGE_FN()
        rc = self.lib.om_solve_global(self.handle, C.byref(self.params), n, float(dt), _p(k), _p(keq),
                                      _p(self.atol_columns),
                                      self.mech.relative_tolerance, _p(y), _p(stats, C.c_int64), len(sizes),
                                      _p(starts, C.c_int32), cb, None, int(total_cells or n))
        if rc:
            raise RuntimeError(self.lib.om_last_error().decode())
        return np.ascontiguousarray(y[:, self.species_columns]), stats

    def backward_euler_global(self, inputs, dt, k=None):
        """Backward Euler on one n-cell State (micm's multi-cell semantics):
        (y_final [n,S] system order, stats [10])."""
        y = np.zeros_like(inputs["concentrations"])
        y[:, self.species_columns] = inputs["concentrations"]
        y = np.ascontiguousarray(y)
        n = len(y)
        k = self._k(inputs) if k is None else np.ascontiguousarray(k)
        stats = np.zeros(10, np.int64)
        rc = self.lib.om_backward_euler_global(self.handle, n, float(dt), _p(k), _p(self.atol_columns),
                                               self.mech.relative_tolerance, _p(y), _p(stats, C.c_int64))
        if rc:
            raise RuntimeError(self.lib.om_last_error().decode())
        return np.ascontiguousarray(y[:, self.species_columns]), stats

    def step_sizes_per_cell(self, inputs, dt, max_steps=512, k=None):
        """Accepted step sizes of each cell's solve: (h [n, max_steps], n_steps [n])."""
        n = len(inputs["temperature"])
        y0 = np.zeros((n, self.S))
        y0[:, self.species_columns] = inputs["concentrations"]
        k = self._k(inputs) if k is None else np.ascontiguousarray(k)
        h = np.zeros((n, max_steps))
        steps = np.zeros(n, np.int32)
        self.lib.om_step_sizes_per_cell(self.handle, C.byref(self.params), n, float(dt), _p(k),
                                        _p(self.atol_columns), self.mech.relative_tolerance, _p(y0), int(max_steps),
                                        _p(h), _p(steps, C.c_int32))
        return h, steps

    def replay_per_cell(self, y0_sys, k, h, n_steps):
        """y0 (system order) advanced by the given accepted step sizes, no error
        control, final clamp: the map the discrete adjoint differentiates."""
        y = np.zeros((len(y0_sys), self.S))
        y[:, self.species_columns] = y0_sys
        h = np.ascontiguousarray(h, np.float64)
        self.lib.om_replay_per_cell(self.handle, C.byref(self.params), len(y), _p(np.ascontiguousarray(k)), _p(h),
                                    _p(np.ascontiguousarray(n_steps, np.int32), C.c_int32), h.shape[1], _p(y))
        return np.ascontiguousarray(y[:, self.species_columns])

    def adjoint_per_cell(self, inputs, dt, ybar_final_sys, threads=0, max_steps=512, k=None):
        """Returns (y_final, dL/dy0, dL/dlogk [n, R input order]) in system order."""
        n, S = len(inputs["temperature"]), self.S
        y0 = np.zeros((n, S))
        y0[:, self.species_columns] = inputs["concentrations"]
        yb = np.zeros((n, S))
        yb[:, self.species_columns] = ybar_final_sys
        k = self._k(inputs) if k is None else np.ascontiguousarray(k)
        yf = np.zeros((n, S)); yb0 = np.zeros((n, S)); kb = np.zeros((n, max(self.R, 1)))
        rc = self.lib.om_adjoint_per_cell(self.handle, C.byref(self.params), n, float(dt), _p(k),
                                          _p(self.atol_columns), self.mech.relative_tolerance, _p(y0), _p(yb),
                                          _p(yf), _p(yb0), _p(kb), int(max_steps),
                                          int(threads or os.cpu_count() or 1))
        if rc:
            raise RuntimeError(self.lib.om_last_error().decode())
        return (yf[:, self.species_columns], yb0[:, self.species_columns],
                kb[:, : self.R][:, self.reaction_columns])
