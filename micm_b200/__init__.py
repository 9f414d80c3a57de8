"""micm_b200 -- a B200-native (sm_100a, FP64) Rosenbrock chemistry solver with
micm's CUDA-path API (NCAR/micm 3.13.0).  See include/micmb.h for the C ABI."""
from .mechanism import (Mechanism, Reaction, arrhenius, branched, reversible, surface, taylor_series,
                        ternary, troe, tunneling, user_defined, ideal_air_density)
from .solver import CompiledMechanism, RosenbrockSolverParameters, Solver, SolverResult, State

__all__ = [
    "Mechanism", "Reaction", "arrhenius", "branched", "reversible", "surface", "taylor_series", "ternary",
    "troe", "tunneling", "user_defined", "ideal_air_density", "CompiledMechanism",
    "RosenbrockSolverParameters", "Solver", "SolverResult", "State",
]
