"""micm_bench's command line over this library (python -m micm_b200.micm_bench):
the keys, messages and result line of test/benchmark/micm_bench.cpp."""
import re

import pytest

from micm_b200 import micm_bench


def run(capsys, *args):
    code = micm_bench.main(["micm_bench", *map(str, args)])
    return code, capsys.readouterr().out


def test_list_has_every_gpu_key(capsys):
    code, out = run(capsys, "list")
    keys = out.split()
    assert code == 0
    assert "ts1/gpu/vector128/in-place/mozart" in keys and "chapman/gpu/vector1/in-place/mozart" in keys
    assert "ts1/gpu-fused/vector8/in-place/mozart" in keys
    assert len(keys) == 2 * 2 * 5


def test_defaults_name_micm_benchs_cpu_case_which_is_not_here(capsys):
    code, out = run(capsys)
    assert code == 1 and "Invalid option combination: chapman/cpu/standard/in-place/mozart" in out


@pytest.mark.parametrize("args", [("abc",), ("10", "x"), ("10", "2", "dt")])
def test_unreadable_arguments(capsys, args):
    code, out = run(capsys, *args)
    assert code == 1 and "Could not read the arguments" in out and "Usage:" in out


def test_unsupported_lu_is_an_invalid_combination(capsys):
    code, out = run(capsys, 100, 2, 30, "gpu", "vector128", "separate", "doolittle", "ts1")
    assert code == 1 and "Invalid option combination: ts1/gpu/vector128/separate/doolittle" in out


def test_without_a_device_the_run_fails_cleanly(capsys):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    code, out = run(capsys, 100, 2, 30, "gpu", "vector128", "in-place", "mozart", "chapman")
    assert code == 1 and out.startswith("Benchmark failed:")


@pytest.mark.gpu
@pytest.mark.parametrize("backend", ["gpu", "gpu-fused"])
def test_result_line(cuda_device, capsys, backend):
    code, out = run(capsys, 1000, 3, 30, backend, "vector128", "in-place", "mozart", "chapman")
    assert code == 0, out
    m = re.match(r"mechanism=chapman backend=(\S+) matrix_type=vector128 lu=mozart/in-place cells=1000 steps=3 "
                 r"dt=30 elapsed_ms=([0-9.]+) ms_per_step=([0-9.]+)", out.strip())
    assert m and m.group(1) == backend and float(m.group(2)) > 0
