"""Whole-solve parity on the GPU against micm's CPU Rosenbrock: final
concentrations within rtol 1e-6 / atol 1e-12 for every cell and species,
accepted-step counts identical in at least 99.9% of cells."""
import numpy as np
import pytest

import oracle
from micm_b200 import synthetic
from micm_b200.mechanism import ideal_air_density

from gpu_helpers import solve_gpu
from mechanisms import all_rate_types, all_rate_types_inputs

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-12


def _close(y, y_ref):
    np.testing.assert_allclose(y, y_ref, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("L", [1, 3, 32, 128])
def test_readme_global(cuda_device, L):
    m = synthetic.readme_mechanism()
    inp = synthetic.cell_inputs(m, 1024, seed=11, readme_foo=(1.0, 30.0))
    ref = oracle.Reference(m, tableau=3)
    y_ref, st_ref = ref.solve_global(inp, 500.0, n_solves=10)
    y, res = solve_gpu(m, inp, 500.0, 3, "plain", "global", n_solves=10, L=L)
    _close(y, y_ref)
    for r, s in zip(res, st_ref):
        assert r.stats["accepted"] == s["accepted"] and r.stats["number_of_steps"] == s["number_of_steps"]
        assert r.stats["function_calls"] == s["function_calls"]
        assert r.stats["jacobian_updates"] == s["jacobian_updates"]


def test_readme_single_cell_table(cuda_device):
    m = synthetic.readme_mechanism()
    T = np.array([287.45]); P = np.array([101319.9])
    inp = dict(temperature=T, pressure=P, air_density=ideal_air_density(P, T),
               concentrations=np.array([[20.0, 0.0, 0.0]]), custom_params=np.zeros((1, 0)))
    y, _ = solve_gpu(m, inp, 500.0, 3, "fused", "per_cell", n_solves=10, L=1)
    assert [float(f"{v:.2e}") for v in y[0]] == [6.13e-02, 1.28e+01, 5.41e+00]


@pytest.mark.parametrize("stages", [2, 3, 4, 40, 60])
def test_tableaus_global(cuda_device, stages):
    m = synthetic.synthetic_mechanism(60, 120, seed=601)
    inp = synthetic.cell_inputs(m, 1, seed=21)
    for k in ("temperature", "pressure", "air_density"):
        inp[k] = np.repeat(inp[k], 40)
    inp["concentrations"] = np.repeat(inp["concentrations"], 40, axis=0) * np.linspace(1, 1.0001, 40)[:, None]
    inp["custom_params"] = np.repeat(inp["custom_params"], 40, axis=0)
    ref = oracle.Reference(m, tableau=stages)
    y_ref, st_ref = ref.solve_global(inp, 600.0)
    y, res = solve_gpu(m, inp, 600.0, stages, "plain", "global", L=16)
    _close(y, y_ref)
    assert res[0].stats["accepted"] == st_ref[0]["accepted"]


@pytest.mark.parametrize("method", ["plain", "fused"])
@pytest.mark.parametrize("name", ["syn60", "syn210", "syn600", "all_kinds"])
def test_per_cell(cuda_device, method, name):
    if name == "all_kinds":
        m, inp, dt, stages = all_rate_types(), all_rate_types_inputs(200, 8), 50.0, 3
    elif name == "syn60":
        m = synthetic.synthetic_mechanism(60, 120, seed=601)
        inp, dt, stages = synthetic.cell_inputs(m, 512, seed=602), 3600.0, 4
    elif name == "syn600":
        # 600 species / 1,500 reactions: the LU factor (11,304 entries) outgrows shared memory
        m = synthetic.CONFIGS["c600"]["mech"]()
        inp, dt, stages = synthetic.cell_inputs(m, 96, seed=6003), 600.0, 4
    else:
        m = synthetic.synthetic_mechanism(210, 440, seed=2101)
        inp, dt, stages = synthetic.cell_inputs(m, 256, seed=2102), 600.0, 4
    ref = oracle.Reference(m, tableau=stages)
    y_ref, st_ref = ref.solve_per_cell(inp, dt)
    y, res = solve_gpu(m, inp, dt, stages, method, "per_cell", L=32)
    np.testing.assert_array_equal(res[0].per_cell_status, st_ref[:, 7])
    _close(y, y_ref)
    same = np.mean(res[0].per_cell_accepted == st_ref[:, 3])
    assert same >= 0.999, same


def test_uneven_day_night(cuda_device):
    m = synthetic.synthetic_mechanism(210, 440, seed=2101)
    inp = synthetic.cell_inputs(m, 384, seed=2103, t_range=(200.0, 310.0), night_fraction=0.5)
    ref = oracle.Reference(m, tableau=4)
    y_ref, st_ref = ref.solve_per_cell(inp, 600.0)
    y, res = solve_gpu(m, inp, 600.0, 4, "fused", "per_cell", L=128)
    _close(y, y_ref)
    assert np.mean(res[0].per_cell_accepted == st_ref[:, 3]) >= 0.999


def test_fused_equals_plain_bitwise(cuda_device):
    m = synthetic.synthetic_mechanism(210, 440, seed=2101)
    inp = synthetic.cell_inputs(m, 200, seed=31)
    y_p, r_p = solve_gpu(m, inp, 600.0, 4, "plain", "per_cell", L=32)
    y_f, r_f = solve_gpu(m, inp, 600.0, 4, "fused", "per_cell", L=32)
    np.testing.assert_array_equal(y_f, y_p)
    np.testing.assert_array_equal(r_f[0].per_cell_accepted, r_p[0].per_cell_accepted)
    for key in ("accepted", "rejected", "number_of_steps", "function_calls", "jacobian_updates", "solves"):
        assert r_f[0].stats[key] == r_p[0].stats[key], key


def test_fused_lu_in_global_memory(cuda_device):
    m = synthetic.synthetic_mechanism(210, 440, seed=2101)
    inp = synthetic.cell_inputs(m, 150, seed=32)
    y_s, _ = solve_gpu(m, inp, 600.0, 4, "fused", "per_cell", L=32)
    y_g, _ = solve_gpu(m, inp, 600.0, 4, "fused", "per_cell", L=32,
                       fused_config=dict(cells_per_cta=4, lu_in_shared=0, variant=1))
    np.testing.assert_array_equal(y_s, y_g)


@pytest.mark.parametrize("config", [dict(variant=1), dict(variant=0, ring_slots=2), dict(variant=0, ring_slots=6),
                                    dict(variant=0, cells_per_cta=1), dict(variant=0, ctas_per_sm=2),
                                    dict(variant=0, lu_in_shared=0, cells_per_cta=10),
                                    dict(variant=0, lu_in_shared=0, cells_per_cta=12, ring_slots=2),
                                    dict(variant=2), dict(variant=2, ctas_per_sm=1),
                                    dict(variant=2, ctas_per_sm=8), dict(variant=2, ctas_per_sm=12)])
def test_fused_variants_bitwise(cuda_device, config):
    """Every fused configuration computes exactly what the plain kernels compute."""
    m = synthetic.synthetic_mechanism(210, 440, seed=2101)
    inp = synthetic.cell_inputs(m, 333, seed=33, t_range=(200.0, 310.0), night_fraction=0.5)
    y_p, r_p = solve_gpu(m, inp, 600.0, 4, "plain", "per_cell", L=32)
    y_f, r_f = solve_gpu(m, inp, 600.0, 4, "fused", "per_cell", L=32, fused_config=config)
    np.testing.assert_array_equal(y_f, y_p)
    np.testing.assert_array_equal(r_f[0].per_cell_accepted, r_p[0].per_cell_accepted)
    assert r_f[0].stats["number_of_steps"] == r_p[0].stats["number_of_steps"]


@pytest.mark.parametrize("config", [dict(variant=0), dict(variant=1), dict(variant=2)])
def test_large_mechanism_variants_bitwise(cuda_device, config):
    """600 species: no streamed schedule (operands beyond 16-bit byte offsets),
    so variant 0 runs the direct kernel; every variant equals the plain path."""
    m = synthetic.CONFIGS["c600"]["mech"]()
    inp = synthetic.cell_inputs(m, 70, seed=6004)
    y_p, r_p = solve_gpu(m, inp, 600.0, 4, "plain", "per_cell", L=32)
    y_f, r_f = solve_gpu(m, inp, 600.0, 4, "fused", "per_cell", L=32, fused_config=config)
    np.testing.assert_array_equal(y_f, y_p)
    np.testing.assert_array_equal(r_f[0].per_cell_accepted, r_p[0].per_cell_accepted)


def test_fused_tiny_and_ragged(cuda_device):
    """Fewer cells than warps, and a cell count that is no multiple of anything."""
    m = synthetic.synthetic_mechanism(60, 120, seed=601)
    for n in (1, 3, 37):
        inp = synthetic.cell_inputs(m, n, seed=40 + n)
        ref = oracle.Reference(m, tableau=4)
        y_ref, st_ref = ref.solve_per_cell(inp, 3600.0)
        y, res = solve_gpu(m, inp, 3600.0, 4, "fused", "per_cell", L=8)
        _close(y, y_ref)
        np.testing.assert_array_equal(res[0].per_cell_accepted, st_ref[:, 3])



@pytest.mark.parametrize("method", ["plain", "fused"])
def test_c2_size_against_micm(cuda_device, method):
    """The 16,384-cell configuration of the 210-species / 440-reaction
    mechanism (4-stage, dt = 600 s, per-cell step control) against micm on all
    host threads (one 1-cell State per cell): every cell and species within
    rtol 1e-6 / atol 1e-12, identical accepted-step counts in at least 99.9 %
    of cells."""
    cfg = synthetic.CONFIGS["c210"]
    mech = cfg["mech"]()
    inp = synthetic.cell_inputs(mech, cfg["cells"], cfg["seed"], **cfg["inputs"])
    y_ref, st_ref = oracle.Reference(mech, tableau=cfg["stages"]).solve_per_cell(inp, cfg["dt"])
    y, res = solve_gpu(mech, inp, cfg["dt"], cfg["stages"], method, "per_cell", L=128)
    _close(y, y_ref)
    assert np.mean(res[0].per_cell_accepted == st_ref[:, 3]) >= 0.999


def test_uneven_1m_workload_sample_against_micm(cuda_device):
    """8,192 cells of the 1,048,576-cell benchmark workload (half night,
    T ~ U(200, 310) K), fused against micm: every species within rtol 1e-6 /
    atol 1e-12, identical accepted-step counts in at least 99.9 % of cells."""
    cfg = synthetic.CONFIGS["c210_uneven"]
    mech = cfg["mech"]()
    inp = synthetic.cell_inputs(mech, 8192, cfg["seed"], **cfg["inputs"])
    y_ref, st_ref = oracle.Reference(mech, tableau=cfg["stages"]).solve_per_cell(inp, cfg["dt"])
    y, res = solve_gpu(mech, inp, cfg["dt"], cfg["stages"], "fused", "per_cell", L=128,
                       fused_config=dict(variant=2, lu_in_shared=0))
    _close(y, y_ref)
    assert np.mean(res[0].per_cell_accepted == st_ref[:, 3]) >= 0.999


@pytest.mark.parametrize("method", ["plain", "fused"])
def test_blocked_schedules_equal_serial_schedules_bitwise(cuda_device, method, monkeypatch):
    """The register-blocked LU and triangular solves (selected by
    MICMB_BLOCKED_SCHEDULES=1 when the solver uploads its tables) against the
    serial schedules: whole per-cell solves, identical bits and step counts."""
    from micm_b200 import Solver
    from gpu_helpers import make_state
    cfg = synthetic.CONFIGS["c210_uneven"]
    mech = cfg["mech"]()
    inp = synthetic.cell_inputs(mech, 1024, cfg["seed"], **cfg["inputs"])
    out = []
    for blocked in (True, False):
        if blocked:
            monkeypatch.setenv("MICMB_BLOCKED_SCHEDULES", "1")
        else:
            monkeypatch.delenv("MICMB_BLOCKED_SCHEDULES", raising=False)
        solver = Solver(mech, cfg["stages"], vector_length=128)
        solver.set_fused_config(variant=2, lu_in_shared=0)
        st = make_state(solver, inp)
        solver.update_state_parameters(st)
        res = solver.solve(cfg["dt"], st, method=method, step_control="per_cell", per_cell=True)
        st.sync_outputs_to_host()
        out.append((st.concentrations(), res.per_cell_accepted))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
