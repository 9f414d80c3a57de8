"""micm_bench's default mechanism, Chapman (test/benchmark/chapman_mechanism.hpp:
9 species, 7 reactions), as ingested from the fixture micm itself wrote
(tests/golden/make_micm_bench.py): numbering equal to micm's state, and the
checkers reproduce micm's results on it.  micm_bench's InitState leaves the
air density at 0 (no reaction here reads it); the fixture keeps that."""
import numpy as np
import pytest

import oracle
from micm_b200 import micm_bench
from micm_b200.solver import CompiledMechanism

GOLDEN = micm_bench.golden("chapman")


def golden_inputs(cols):
    return dict(temperature=GOLDEN["temperature"], pressure=GOLDEN["pressure"], air_density=GOLDEN["air_density"],
                concentrations=np.ascontiguousarray(GOLDEN["initial_variables"][:, cols]),
                custom_params=np.ascontiguousarray(GOLDEN["custom_parameters"]))


def test_numbering_equals_micm_state():
    mech = micm_bench.mechanism("chapman")
    cm = CompiledMechanism(mech)
    cols = micm_bench.micm_columns("chapman")
    assert mech.n_species == 9 and mech.n_reactions == 7
    np.testing.assert_array_equal(cm.species_columns, [cols["species"][s] for s in mech.species])
    labels = mech.custom_param_labels()
    np.testing.assert_array_equal([cols["custom_parameters"][l] for l in labels], np.arange(len(labels)))


def test_inputs_follow_the_benchmark_state():
    mech = micm_bench.mechanism("chapman")
    inp = micm_bench.inputs("chapman", 2)
    cols = CompiledMechanism(mech).species_columns
    np.testing.assert_array_equal(inp["concentrations"][0], GOLDEN["initial_variables"][0, cols])
    np.testing.assert_array_equal(inp["custom_params"][0], GOLDEN["custom_parameters"][0])
    assert inp["air_density"][0] == 0.0


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
def test_restatement_rate_constants_equal_micm():
    mech = micm_bench.mechanism("chapman")
    R = oracle.Restatement(mech, tableau_kind=micm_bench.TABLEAU)
    inp = golden_inputs(R.species_columns)
    k = R.rate_constants(inp["temperature"], inp["pressure"], inp["air_density"], inp["custom_params"])
    np.testing.assert_allclose(k, GOLDEN["rate_constants"], rtol=1e-14, atol=0)


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_flattened_mechanism_reproduces_micm_from_its_header():
    mech = micm_bench.mechanism("chapman")
    ref = oracle.Reference(mech, tableau=micm_bench.TABLEAU)
    inp = golden_inputs(ref.species_columns)
    for s in range(len(GOLDEN["variables"])):
        y, stats = ref.solve_global(inp, float(GOLDEN["dt"]))
        np.testing.assert_array_equal(ref.y_to_columns(y), GOLDEN["variables"][s])
        assert stats[0]["accepted"] == GOLDEN["stats"][s, 0]
        inp = dict(inp, concentrations=y)


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
def test_restatement_per_cell_on_varied_cells_equals_micm():
    mech = micm_bench.mechanism("chapman")
    inp = micm_bench.inputs("chapman", 64, seed=21)
    R = oracle.Restatement(mech, tableau_kind=micm_bench.TABLEAU)
    y, st = R.solve_per_cell(inp, micm_bench.DT)
    if oracle.reference_available():
        y_ref, st_ref = oracle.Reference(mech, tableau=micm_bench.TABLEAU).solve_per_cell(inp, micm_bench.DT)
        np.testing.assert_array_equal(st[:, 3], st_ref[:, 3])
        np.testing.assert_allclose(y, y_ref, rtol=1e-12, atol=1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("L", [1, 4, 32])
def test_gpu_global_solves_match_micm(cuda_device, L):
    from micm_b200 import Solver
    from gpu_helpers import make_state
    mech = micm_bench.mechanism("chapman")
    solver = Solver(mech, micm_bench.TABLEAU, vector_length=L)
    cols = solver.compiled.species_columns
    st = make_state(solver, golden_inputs(cols))
    solver.update_state_parameters(st)
    np.testing.assert_allclose(st.rate_constants(), GOLDEN["rate_constants"], rtol=1e-12, atol=0)
    for s in range(len(GOLDEN["variables"])):
        res = solver.solve(float(GOLDEN["dt"]), st, method="plain", step_control="global")
        st.sync_outputs_to_host()
        np.testing.assert_allclose(st.concentrations(), GOLDEN["variables"][s][:, cols], rtol=1e-6, atol=1e-12)
        assert res.stats["accepted"] == GOLDEN["stats"][s, 0]


@pytest.mark.gpu
@pytest.mark.parametrize("method,config", [("plain", None), ("fused", dict(variant=0)), ("fused", dict(variant=2))])
def test_gpu_per_cell_varied_cells_match_micm(cuda_device, method, config):
    from gpu_helpers import solve_gpu
    mech = micm_bench.mechanism("chapman")
    inp = micm_bench.inputs("chapman", 256, seed=21)
    y_ref, st_ref = oracle.Reference(mech, tableau=micm_bench.TABLEAU).solve_per_cell(inp, micm_bench.DT)
    y, res = solve_gpu(mech, inp, micm_bench.DT, micm_bench.TABLEAU, method, "per_cell", L=32, fused_config=config)
    np.testing.assert_allclose(y, y_ref, rtol=1e-6, atol=1e-12)
    assert np.mean(res[0].per_cell_accepted == st_ref[:, 3]) >= 0.999
