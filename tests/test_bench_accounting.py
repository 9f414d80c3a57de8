"""bench.py's roofline accounting on the host: the compulsory bytes per
operation of the formulation with working sets in HBM (bytes_per_solve_unit)
and the FP64 operation counts (flops_per_solve_unit) for the 210-species
benchmark mechanism, the figures the benchmark line divides by its kernel
time."""
import os
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from micm_b200 import synthetic  # noqa: E402
from micm_b200.solver import CompiledMechanism  # noqa: E402


@pytest.fixture(scope="module")
def c210():
    mech = synthetic.CONFIGS["c210_uneven"]["mech"]()
    return mech, types.SimpleNamespace(compiled=CompiledMechanism(mech))


def test_compulsory_bytes_per_attempt(c210):
    mech, solver = c210
    u = bench.bytes_per_solve_unit(mech, solver, 4)
    S, R, nnz = 210, 440, 2596
    assert u["jac"] == 24 * nnz and u["lu"] == 8 * (2 * nnz + 2 * S) and u["solve"] == 8 * (nnz + 2 * S)
    assert u["force"] == 8 * (R + 3 * S)
    # one attempt of the 4-stage tableau: -J, LU, 4 solves, 3 forcing evaluations, stage sums and error norm
    per_attempt = u["jac"] + u["lu"] + 4 * u["solve"] + 3 * u["force"] + u["attempt"]
    assert 300e3 < per_attempt < 315e3


def test_solve_bytes_and_flops_scale_with_statistics(c210):
    mech, solver = c210
    u = bench.bytes_per_solve_unit(mech, solver, 4)
    f = bench.flops_per_solve_unit(mech, solver, 4)
    stats = dict(function_calls=3, jacobian_updates=1, decompositions=1, solves=4, number_of_steps=1)
    one = bench.solve_bytes(u, stats)
    two = bench.solve_bytes(u, {k: 2 * v for k, v in stats.items()})
    assert two == 2 * one
    assert f["lu"] == 2 * 7992 + 1155 + 210
    assert bench.solve_flops(f, stats) > 0


def test_job_throughput_counts_every_rank():
    assert bench.job_throughput(1000, 4, 2, 0.5) == 1000 * 4 * 2 / 0.5
