"""Python mirror of micm's CUDA-path API over the C ABI.

    solver = Solver(mechanism, RosenbrockSolverParameters.four_stage(), vector_length=128)
    state = solver.get_state(n_cells)
    state.conditions ...; state[species] = values
    state.sync_inputs_to_device()
    solver.update_state_parameters(state)
    result = solver.solve(dt, state)            # plain kernels, micm's single step size
    result = solver.solve(dt, state, method="fused", step_control="per_cell")
    state.sync_outputs_to_host()

mirrors CudaSolverBuilderInPlace<...>::Build, Solver::GetState,
Solver::UpdateStateParameters, Solver::Solve and CudaState::Sync*
(include/micm/cuda/solver/cuda_solver_builder.hpp:25-37,
include/micm/solver/solver.hpp:133-247, include/micm/cuda/solver/cuda_state.hpp:132-148).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Dict, Optional, Union

import numpy as np

from . import _native
from ._abi import BackwardEulerParams, DescHolder, FusedConfig, MechanismInfo, RosenbrockParams, SolverStats
from ._native import check, lib
from .mechanism import Mechanism, from_vector_layout, padded_cells, to_vector_layout

BUF_VARIABLES = 0
BUF_CUSTOM_PARAMS = 1
BUF_RATE_CONSTANTS = 2
BUF_JACOBIAN = 3
BUF_CONDITIONS = 4
BUF_ABSOLUTE_TOLERANCE = 5
BUF_FORCING = 6
BUF_SCRATCH_Y = 7

METHODS = {"plain": 0, "fused": 1}
STEP_CONTROL = {"global": 0, "per_cell": 1}

# micm::SolverState
SOLVER_STATES = {0: "NotYetCalled", 1: "Running", 2: "Converged", 3: "ConvergenceExceededMaxSteps",
                 4: "StepSizeTooSmall", 5: "RepeatedlySingularMatrix", 6: "NaNDetected", 7: "InfDetected"}
CONVERGED = 2


def _f64(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i32(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class RosenbrockSolverParameters:
    """RosenbrockSolverParameters::*Parameters() (rosenbrock_solver_parameters.hpp:152-434)."""

    @staticmethod
    def _make(kind: int) -> RosenbrockParams:
        p = RosenbrockParams()
        check(lib().micmb_rosenbrock_params_default(kind, C.byref(p)))
        return p

    two_stage = staticmethod(lambda: RosenbrockSolverParameters._make(2))
    three_stage = staticmethod(lambda: RosenbrockSolverParameters._make(3))
    four_stage = staticmethod(lambda: RosenbrockSolverParameters._make(4))
    four_stage_differential_algebraic = staticmethod(lambda: RosenbrockSolverParameters._make(40))
    six_stage_differential_algebraic = staticmethod(lambda: RosenbrockSolverParameters._make(60))

    @staticmethod
    def from_stages(stages: int) -> RosenbrockParams:
        return RosenbrockSolverParameters._make({2: 2, 3: 3, 4: 4, 40: 40, 60: 60}[stages])


class CompiledMechanism:
    """micmb_mechanism: the host-side symbolic compile (no GPU needed)."""

    def __init__(self, mech: Mechanism):
        self.mech = mech
        self._desc = DescHolder(mech.flat())
        h = C.c_void_p()
        check(lib().micmb_mechanism_create(C.byref(self._desc.desc), C.byref(h)))
        self.handle = h
        info = MechanismInfo()
        check(lib().micmb_mechanism_get_info(self.handle, C.byref(info)))
        self.info = info.as_dict()
        S, R = mech.n_species, mech.n_reactions
        self.species_columns = np.zeros(S, np.int32)
        check(lib().micmb_mechanism_species_columns(self.handle, _i32(self.species_columns)))
        self.reaction_columns = np.zeros(max(R, 1), np.int32)[:R]
        if R:
            check(lib().micmb_mechanism_reaction_columns(self.handle, _i32(self.reaction_columns)))
        self.param_columns = np.zeros(max(R, 1), np.int32)[:R]
        if R:
            check(lib().micmb_mechanism_custom_param_columns(self.handle, _i32(self.param_columns)))
        nnz = self.info["jacobian_nnz"]
        self.rows = np.zeros(nnz, np.int32)
        self.cols = np.zeros(nnz, np.int32)
        check(lib().micmb_mechanism_jacobian_pattern(self.handle, _i32(self.rows), _i32(self.cols)))
        nu = self.info["jacobian_nnz_unfilled"]
        self.rows_unfilled = np.zeros(nu, np.int32)
        self.cols_unfilled = np.zeros(nu, np.int32)
        check(lib().micmb_mechanism_jacobian_pattern_unfilled(self.handle, _i32(self.rows_unfilled),
                                                              _i32(self.cols_unfilled)))
        self.hash = int(lib().micmb_mechanism_hash(self.handle))

    def stream_stats(self) -> Dict[str, Dict[str, int]]:
        """Blocks, segments, lane steps and terms of each streamed phase."""
        out = np.zeros(28, np.int64)
        check(lib().micmb_mechanism_stream_stats(self.handle, out.ctypes.data_as(C.POINTER(C.c_int64))))
        names = ["forcing", "jacobian", "lu", "forward", "backward", "forward_t", "backward_t"]
        return {n: dict(blocks=int(out[4 * i]), segments=int(out[4 * i + 1]), steps=int(out[4 * i + 2]),
                        terms=int(out[4 * i + 3])) for i, n in enumerate(names)}

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and h.value and _native._lib is not None:
                _native._lib.micmb_mechanism_destroy(h)
                self.handle = None
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass


@dataclasses.dataclass
class SolverResult:
    """micm::SolverResult (solver_result.hpp:77-83) summed over cells."""
    state: int
    stats: Dict[str, float]
    per_cell_status: Optional[np.ndarray] = None
    per_cell_accepted: Optional[np.ndarray] = None

    @property
    def converged(self) -> bool:
        return self.state == CONVERGED


class Solver:
    def __init__(self, mech: Union[Mechanism, CompiledMechanism],
                 params: Union[int, RosenbrockParams, None] = None, vector_length: int = 128):
        self.compiled = mech if isinstance(mech, CompiledMechanism) else CompiledMechanism(mech)
        self.mech = self.compiled.mech
        if params is None:
            params = RosenbrockSolverParameters.three_stage()
        elif isinstance(params, int):
            params = RosenbrockSolverParameters.from_stages(params)
        self.params = params
        self.vector_length = int(vector_length)
        h = C.c_void_p()
        check(lib().micmb_solver_create(self.compiled.handle, C.byref(self.params), C.byref(h)))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and h.value and _native._lib is not None:
                _native._lib.micmb_solver_destroy(h)
                self.handle = None
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass

    def set_rate_scale(self, scale: np.ndarray):
        scale = np.ascontiguousarray(scale, dtype=np.float64)
        assert scale.shape == (self.mech.n_reactions,)
        check(lib().micmb_solver_set_rate_scale(self.handle, _f64(scale)))

    def set_fused_config(self, cells_per_cta=0, lu_in_shared=1, ctas_per_sm=0, ring_slots=0, variant=0):
        """variant 0: TMA-streamed warp-specialised kernel; 1: direct kernel (warp per cell);
        2: one cell per thread, working sets in global memory."""
        cfg = FusedConfig(int(cells_per_cta), int(lu_in_shared), int(ctas_per_sm), int(ring_slots), int(variant))
        check(lib().micmb_solver_set_fused_config(self.handle, C.byref(cfg)))

    def get_fused_config(self) -> Dict[str, int]:
        cfg = FusedConfig()
        check(lib().micmb_solver_get_fused_config(self.handle, C.byref(cfg)))
        return dict(cells_per_cta=cfg.cells_per_cta, lu_in_shared=cfg.lu_in_shared,
                    ctas_per_sm=cfg.ctas_per_sm, ring_slots=cfg.ring_slots, variant=cfg.variant)

    def get_state(self, n_cells: int = 1, vector_length: Optional[int] = None) -> "State":
        return State(self, n_cells, vector_length or self.vector_length)

    def update_state_parameters(self, state: "State"):
        check(lib().micmb_update_state_parameters(self.handle, state.handle))

    def solve(self, dt: float, state: "State", method: str = "plain", step_control: str = "global",
              per_cell: bool = False) -> SolverResult:
        stats = SolverStats()
        n = state.n_cells
        pst = np.zeros(max(n, 1), np.int32) if per_cell else None
        pac = np.zeros(max(n, 1), np.int32) if per_cell else None
        check(lib().micmb_solve(self.handle, state.handle, float(dt), METHODS[method], STEP_CONTROL[step_control],
                                C.byref(stats), _i32(pst) if per_cell else None,
                                _i32(pac) if per_cell else None))
        return SolverResult(stats.state, stats.as_dict(), pst[:n] if per_cell else None,
                            pac[:n] if per_cell else None)

    def solve_backward_euler(self, dt: float, state: "State", step_control: str = "global",
                             params: Optional[BackwardEulerParams] = None, per_cell: bool = False) -> SolverResult:
        """micm's Backward Euler Solve (backward_euler.inl:10-186) on the GPU.  "global": one
        step size and convergence test for all cells (micm's multi-cell State); "per_cell": each
        cell as a 1-cell State.  params: micm's defaults when None."""
        stats = SolverStats()
        n = state.n_cells
        pst = np.zeros(max(n, 1), np.int32) if per_cell else None
        pac = np.zeros(max(n, 1), np.int32) if per_cell else None
        check(lib().micmb_solve_backward_euler(self.handle, state.handle, float(dt),
                                               C.byref(params) if params is not None else None,
                                               STEP_CONTROL[step_control], C.byref(stats),
                                               _i32(pst) if per_cell else None, _i32(pac) if per_cell else None))
        return SolverResult(stats.state, stats.as_dict(), pst[:n] if per_cell else None,
                            pac[:n] if per_cell else None)

    @staticmethod
    def backward_euler_params() -> BackwardEulerParams:
        """micm's default Backward Euler parameters (a ctypes struct the caller may edit)."""
        p = BackwardEulerParams()
        check(lib().micmb_backward_euler_params_default(C.byref(p)))
        return p

    def autotune(self, dt: float, state: "State", cache_path: Optional[str] = None) -> Dict[str, int]:
        """Time the fused configurations on this state and keep the fastest."""
        cfg = FusedConfig()
        check(lib().micmb_autotune(self.handle, state.handle, float(dt),
                                   cache_path.encode() if cache_path else None, C.byref(cfg)))
        return self.get_fused_config()

    def solve_graph(self, dt: float, state: "State", n_repeats: int):
        """n_repeats x (update_state_parameters + fused per-cell solve) from one CUDA graph."""
        check(lib().micmb_solve_graph(self.handle, state.handle, float(dt), int(n_repeats)))

    def set_adjoint_memory_limit(self, n_bytes: int):
        """Device bytes solve_adjoint may hold in checkpoints (0: 80% of the free device memory).
        Cells are solved and swept in chunks that fit; results do not depend on the chunking."""
        check(lib().micmb_set_adjoint_memory_limit(self.handle, int(n_bytes)))

    def solve_adjoint(self, dt: float, state: "State", dloss_dy_final: np.ndarray, max_checkpoints: int = 256):
        """Returns (dL/dy0 [n, S] state columns, dL/dlog k [R] input order, SolverResult)."""
        n, S, L = state.n_cells, self.mech.n_species, state.L
        g = to_vector_layout(np.asarray(dloss_dy_final, np.float64), L)
        dy0 = np.zeros_like(g)
        dk = np.zeros(max(self.mech.n_reactions, 1))
        stats = SolverStats()
        check(lib().micmb_solve_adjoint(self.handle, state.handle, float(dt), _f64(g), _f64(dy0), _f64(dk),
                                        int(max_checkpoints), C.byref(stats)))
        return (from_vector_layout(dy0, n, S, L), dk[: self.mech.n_reactions],
                SolverResult(stats.state, stats.as_dict()))


class State:
    """Host mirror + device buffers of one CudaState (n_cells, vector length L)."""

    def __init__(self, solver: Solver, n_cells: int, L: int):
        self.solver = solver
        self.n_cells = int(n_cells)
        self.L = int(L)
        mech = solver.mech
        self.S = mech.n_species
        self.P = solver.compiled.info["n_custom_params"]
        self.R = mech.n_reactions
        h = C.c_void_p()
        check(lib().micmb_state_create(solver.handle, self.n_cells, self.L, C.byref(h)))
        self.handle = h
        cols = solver.compiled.species_columns
        self.variable_map = {name: int(cols[i]) for i, name in enumerate(mech.species)}
        self.custom_rate_parameter_map = {lab: i for i, lab in enumerate(mech.custom_param_labels())}
        self.variables = np.zeros((self.n_cells, self.S))
        self.custom_rate_parameters = np.zeros((self.n_cells, self.P))
        self.temperature = np.zeros(self.n_cells)
        self.pressure = np.zeros(self.n_cells)
        self.air_density = np.zeros(self.n_cells)
        self.relative_tolerance = mech.relative_tolerance
        self.absolute_tolerance = np.zeros(self.S)
        self.absolute_tolerance[cols] = mech.atol()

    def __del__(self):
        h = getattr(self, "handle", None)
        try:
            if h and h.value and _native._lib is not None:
                _native._lib.micmb_state_destroy(h)
                self.handle = None
        except (AttributeError, TypeError):  # interpreter shutdown: the library is already unloaded
            pass

    # micm State::operator[](species) / SetConcentrations in system order
    def set_concentrations(self, y_system_order: np.ndarray):
        self.variables[:, self.solver.compiled.species_columns] = y_system_order

    def concentrations(self) -> np.ndarray:
        return self.variables[:, self.solver.compiled.species_columns].copy()

    def set_custom_rate_parameters(self, params_label_order: np.ndarray):
        if self.P:
            self.custom_rate_parameters[:, :] = params_label_order

    def set_conditions(self, temperature, pressure, air_density):
        self.temperature[:] = temperature
        self.pressure[:] = pressure
        self.air_density[:] = air_density

    def set_inputs(self, inputs: Dict[str, np.ndarray]):
        self.set_conditions(inputs["temperature"], inputs["pressure"], inputs["air_density"])
        self.set_concentrations(inputs["concentrations"])
        if self.P:
            self.set_custom_rate_parameters(inputs["custom_params"])

    def set_global_exchange(self, allgather, world: int, total_cells: int):
        """Make global-step-control solves of this state one shard of a job over
        `world` ranks.  allgather(send_ptr, recv_ptr, world, stream_ptr) -> int
        queues, on the CUDA stream, an all-gather of one double per rank from
        device address send_ptr into recv_ptr[0:world] in rank order.  None
        restores the single-GPU solve."""
        from ._native import ALLGATHER_FN
        if allgather is None:
            self._gx = None
            check(lib().micmb_state_set_global_exchange(self.handle, ALLGATHER_FN(), None, 1, 0))
            return
        def trampoline(send, recv, w, stream, _user):
            try:
                return int(allgather(send, recv, w, stream) or 0)
            except Exception:  # an exception must not cross the C ABI
                return -1
        self._gx = ALLGATHER_FN(trampoline)  # kept alive as long as the state
        check(lib().micmb_state_set_global_exchange(self.handle, self._gx, None, int(world), int(total_cells)))

    def upload(self, buffer: int, host_vector_layout: np.ndarray):
        a = np.ascontiguousarray(host_vector_layout, dtype=np.float64)
        check(lib().micmb_state_upload(self.handle, buffer, _f64(a)))

    def download(self, buffer: int, count: int) -> np.ndarray:
        a = np.zeros(count)
        check(lib().micmb_state_download(self.handle, buffer, _f64(a)))
        return a

    def device_buffer(self, buffer: int):
        p = C.POINTER(C.c_double)()
        n = C.c_int64()
        check(lib().micmb_state_device_buffer(self.handle, buffer, C.byref(p), C.byref(n)))
        return C.cast(p, C.c_void_p).value, n.value

    def sync_inputs_to_device(self):
        """Variables, conditions, custom parameters and tolerances to the GPU."""
        L = self.L
        self.upload(BUF_VARIABLES, to_vector_layout(self.variables, L))
        cond = np.stack([self.temperature, self.pressure, self.air_density], axis=1)
        self.upload(BUF_CONDITIONS, to_vector_layout(cond, L))
        if self.P:
            self.upload(BUF_CUSTOM_PARAMS, to_vector_layout(self.custom_rate_parameters, L))
        self.upload(BUF_ABSOLUTE_TOLERANCE, self.absolute_tolerance)
        check(lib().micmb_state_set_relative_tolerance(self.handle, float(self.relative_tolerance)))

    def sync_outputs_to_host(self):
        npad = padded_cells(self.n_cells, self.L)
        buf = self.download(BUF_VARIABLES, npad * self.S)
        self.variables[:, :] = from_vector_layout(buf, self.n_cells, self.S, self.L)

    def rate_constants(self) -> np.ndarray:
        npad = padded_cells(self.n_cells, self.L)
        return from_vector_layout(self.download(BUF_RATE_CONSTANTS, npad * self.R), self.n_cells, self.R, self.L)

    def jacobian(self) -> np.ndarray:
        npad = padded_cells(self.n_cells, self.L)
        nnz = self.solver.compiled.info["jacobian_nnz"]
        return from_vector_layout(self.download(BUF_JACOBIAN, npad * nnz), self.n_cells, nnz, self.L)
