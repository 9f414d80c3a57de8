"""micm's CUDA-path C++ API (include/micm_b200/micm.hpp) over the C ABI."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "micm_b200")

README_TABLE = [
    "0,   1.18e+01,   5.90e+00,   1.91e+00", "500,   6.79e+00,   9.05e+00,   3.32e+00",
    "1000,   3.83e+00,   1.07e+01,   4.21e+00", "1500,   2.14e+00,   1.17e+01,   4.74e+00",
    "2000,   1.19e+00,   1.22e+01,   5.04e+00", "2500,   6.58e-01,   1.24e+01,   5.21e+00",
    "3000,   3.64e-01,   1.26e+01,   5.31e+00", "3500,   2.01e-01,   1.27e+01,   5.36e+00",
    "4000,   1.11e-01,   1.27e+01,   5.39e+00", "4500,   6.13e-02,   1.28e+01,   5.41e+00",
]


@pytest.fixture(scope="module")
def readme_binary(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "readme_example")
    subprocess.run(["g++", "-std=c++20", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "readme_example.cpp"), "-o", out, "-L" + LIB_DIR,
                    "-lmicmb", "-Wl,-rpath," + LIB_DIR], check=True)
    return out


def _has_gpu():
    import torch
    return torch.cuda.is_available()


def test_cpp_api_compiles_and_reports_missing_device(readme_binary):
    if _has_gpu():
        pytest.skip("a GPU is present; covered by the gpu test")
    r = subprocess.run([readme_binary], capture_output=True, text=True)
    assert r.returncode == 3 and "no CUDA device" in r.stderr


def _rows(stdout):
    return [re.sub(r"\s+", " ", l.strip()) for l in stdout.strip().splitlines()[1:]]


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["plain", "fused"])
def test_cpp_readme_example_on_gpu(cuda_device, readme_binary, method):
    r = subprocess.run([readme_binary, method], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert _rows(r.stdout) == [re.sub(r"\s+", " ", l) for l in README_TABLE]


# micm's source tree, when the caller names it (MICM_REFERENCE=<micm source tree>)
REFERENCE_BENCHMARK = os.path.join(os.environ.get("MICM_REFERENCE", ""), "test", "benchmark")


@pytest.mark.skipif(not os.environ.get("MICM_REFERENCE")
                    or not os.path.exists(os.path.join(REFERENCE_BENCHMARK, "ts1_mechanism.hpp")),
                    reason="micm's benchmark sources are not given (MICM_REFERENCE)")
def test_micm_benchmark_mechanisms_build_unchanged(tmp_path):
    """micm's own benchmark mechanisms (TS1, Chapman: test/benchmark/*_mechanism.hpp)
    compile unchanged against this library's C++ API (include/micm/GPU.hpp,
    CPU.hpp, util/property_keys.hpp serve micm's include names), link to
    libmicmb.so and run up to the device (exit 3 without one)."""
    out = str(tmp_path / "micm_bench_mechanisms")
    subprocess.run(["g++", "-std=c++20", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + REFERENCE_BENCHMARK,
                    os.path.join(ROOT, "tests", "cpp", "micm_bench_mechanisms.cpp"), "-o", out, "-L" + LIB_DIR,
                    "-lmicmb", "-Wl,-rpath," + LIB_DIR], check=True)
    if not _has_gpu():
        r = subprocess.run([out], capture_output=True, text=True)
        assert r.returncode == 3 and "no CUDA device" in r.stderr


@pytest.fixture(scope="module")
def dae_binary(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "dae_example")
    subprocess.run(["g++", "-std=c++20", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dae_example.cpp"), "-o", out, "-L" + LIB_DIR,
                    "-lmicmb", "-Wl,-rpath," + LIB_DIR], check=True)
    return out


def test_cpp_constraints_api_compiles(dae_binary):
    """micm's SetConstraints / EquilibriumConstraint / Constraint spelling builds
    against micm.hpp (and reports the missing device without a GPU)."""
    if _has_gpu():
        pytest.skip("a GPU is present; covered by the gpu test")
    r = subprocess.run([dae_binary], capture_output=True, text=True)
    assert r.returncode == 3 and "no CUDA device" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["plain", "fused"])
def test_cpp_constraints_on_gpu_equal_restatement(cuda_device, dae_binary, method):
    """The C++ DAE example (3 cells, equilibrium constraint started off
    equilibrium) equals the restatement of micm's DAE Rosenbrock in its
    correctly rounded mode bit for bit: global step control for "plain",
    per-cell for "fused"."""
    import sys
    import numpy as np
    sys.path.insert(0, ROOT)
    import oracle
    from dae_cases import equilibrium, equilibrium_inputs
    r = subprocess.run([dae_binary, method], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    m = equilibrium()
    inp = equilibrium_inputs(m, 3, False)
    inp["temperature"] = np.array([280.0, 295.0, 310.0])
    from micm_b200.mechanism import ideal_air_density
    inp["air_density"] = ideal_air_density(inp["pressure"], inp["temperature"])
    R = oracle.Restatement(m, tableau_kind=40, correctly_rounded=True)
    y = inp["concentrations"]
    t = 0.0
    rows = [l.split() for l in r.stdout.strip().splitlines()]
    assert [float(row[0]) for row in rows] == [1.0, 5.0, 20.0, 60.0]
    for row in rows:
        target = float(row[0])
        if method == "plain":
            y, st = R.solve_global(dict(inp, concentrations=y), target - t)
            iters = st[9]
        else:
            y, st = R.solve_per_cell(dict(inp, concentrations=y), target - t, threads=1)
            iters = st[:, 9].sum()
        assert int(row[1]) == iters
        np.testing.assert_array_equal(np.array([float(v) for v in row[2:]]).reshape(3, 3), y)
        t = target


def test_cpp_constraint_validation(tmp_path):
    """micm.hpp's constraint classes and builder reject invalid constraints
    with MicmException before any device call (CPU)."""
    out = str(tmp_path / "constraint_errors")
    subprocess.run(["g++", "-std=c++20", "-O1", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "constraint_errors.cpp"), "-o", out, "-L" + LIB_DIR,
                    "-lmicmb", "-Wl,-rpath," + LIB_DIR], check=True)
    r = subprocess.run([out], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(" ok") == 6, r.stdout


def test_c_abi_dae_mechanism_pattern_equals_micms(tmp_path):
    """A DAE mechanism built through the plain C description (gcc, micmb.h
    only): its LU-filled Jacobian pattern equals micm's for the same system
    (micm built here, SetConstraints)."""
    import sys
    import numpy as np
    sys.path.insert(0, ROOT)
    import oracle
    if not oracle.reference_available():
        pytest.skip("oracle/_ref not built")
    from dae_cases import equilibrium
    out = str(tmp_path / "dae_c_api")
    subprocess.run(["gcc", "-std=c11", "-O1", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dae_c_api.c"), "-o", out, "-L" + LIB_DIR, "-lmicmb",
                    "-Wl,-rpath," + LIB_DIR], check=True)
    r = subprocess.run([out], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    nnz = int(lines[0].split()[1])
    pairs = np.array([[int(v) for v in l.split()] for l in lines[1:]])
    assert len(pairs) == nnz
    ref = oracle.Reference(equilibrium(), tableau=40)
    np.testing.assert_array_equal(pairs[:, 0], ref.rows)
    np.testing.assert_array_equal(pairs[:, 1], ref.cols)
