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


@pytest.mark.skipif(not __import__("oracle").reference_available(), reason="oracle/_ref not built")
def test_reference_arm_prints_its_contract_line():
    """`bench.py --impl reference` (micm on the host cores) on a small sample:
    one JSON line with the contract's keys, its own e2e and cpu_baseline."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--cells", "2048", "--cpu-sample", "256",
                        "--steps", "1", "--warmup", "1"], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
