"""micm's TS1 benchmark mechanism (test/benchmark/ts1_mechanism.hpp) as
ingested from the fixture micm itself wrote (tests/golden/make_micm_bench.py): the
numbering equals micm's state, and the checkers reproduce micm's results on it."""
import numpy as np
import pytest

import oracle
from micm_b200 import ts1
from micm_b200.solver import CompiledMechanism

GOLDEN = np.load(ts1.FIXTURE.replace("ts1_mechanism.json", "ts1_micm.npz"))


def _golden_inputs(mech, cols):
    y_sys = GOLDEN["initial_variables"][:, cols]
    return dict(temperature=GOLDEN["temperature"], pressure=GOLDEN["pressure"], air_density=GOLDEN["air_density"],
                concentrations=np.ascontiguousarray(y_sys),
                custom_params=np.ascontiguousarray(GOLDEN["custom_parameters"]))


def test_numbering_equals_micm_state():
    mech = ts1.mechanism()
    cm = CompiledMechanism(mech)
    cols = ts1.micm_columns()
    assert mech.n_species == 209 and mech.n_reactions == 547
    np.testing.assert_array_equal(cm.species_columns, [cols["species"][s] for s in mech.species])
    # custom parameters: label order is micm's column order
    labels = mech.custom_param_labels()
    np.testing.assert_array_equal([cols["custom_parameters"][l] for l in labels], np.arange(len(labels)))
    # LU statistics micm reports for TS1 (2,381 filled nonzeros, 6,986 updates, 1,244 multipliers)
    assert cm.info["jacobian_nnz"] == 2381
    assert cm.info["lu_updates"] == 6986
    assert cm.info["lu_lower"] == 1244


def test_inputs_follow_the_benchmark_state():
    mech = ts1.mechanism()
    inp = ts1.inputs(3)
    cols = CompiledMechanism(mech).species_columns
    np.testing.assert_array_equal(inp["concentrations"][0], GOLDEN["initial_variables"][0, cols])
    np.testing.assert_array_equal(inp["custom_params"][0], GOLDEN["custom_parameters"][0])
    assert inp["temperature"][0] == GOLDEN["temperature"][0]
    varied = ts1.inputs(16, seed=3)
    assert np.all(varied["concentrations"] >= 0) and varied["temperature"].std() > 1.0


@pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
def test_restatement_rate_constants_equal_micm():
    mech = ts1.mechanism()
    R = oracle.Restatement(mech, tableau_kind=ts1.TABLEAU)
    inp = _golden_inputs(mech, R.species_columns)
    k = R.rate_constants(inp["temperature"], inp["pressure"], inp["air_density"], inp["custom_params"])
    # both in micm's rate-constant columns (reactions after micm's type sort)
    np.testing.assert_allclose(k, GOLDEN["rate_constants"], rtol=1e-14, atol=0)


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_flattened_mechanism_reproduces_micm_from_its_header():
    """micm built from the flattened description (oracle/_ref) gives what micm
    built from its own header gave: 10 global Solve(30 s) on 4 varied cells."""
    mech = ts1.mechanism()
    ref = oracle.Reference(mech, tableau=ts1.TABLEAU)
    inp = _golden_inputs(mech, ref.species_columns)
    for s in range(len(GOLDEN["variables"])):
        y, stats = ref.solve_global(inp, float(GOLDEN["dt"]))
        np.testing.assert_array_equal(ref.y_to_columns(y), GOLDEN["variables"][s])
        assert stats[0]["accepted"] == GOLDEN["stats"][s, 0]
        assert stats[0]["number_of_steps"] == GOLDEN["stats"][s, 2]
        inp = dict(inp, concentrations=y)


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_vector128_groups_solve_identical_cells_like_per_cell():
    """The CPU baseline's micm_bench layout (vector ordering L = 128, one State
    per 128 cells) takes the same steps as per-cell States on identical cells;
    values agree within the solve's own absolute tolerance (1e-3, micm's
    default, which micm_bench uses)."""
    mech = ts1.mechanism()
    ref = oracle.Reference(mech, tableau=ts1.TABLEAU)
    inp = ts1.inputs(256)
    y1, s1 = ref.solve_per_cell(inp, ts1.DT)
    y2, s2 = ref.solve_groups_v128(inp, ts1.DT, group=128)
    assert len(s2) == 2
    for g in s2:
        assert g[2] == s1[0, 2] and g[3] == s1[0, 3]      # number_of_steps, accepted
    np.testing.assert_allclose(y2, y1, rtol=1e-6, atol=1e-3)


def test_json_description_round_trips():
    """mechanism_to_dict / mechanism_from_dict keep every field micm's numbering and the kernels use."""
    from micm_b200.mechanism import mechanism_from_dict, mechanism_to_dict
    from mechanisms import all_rate_types
    for m in (ts1.mechanism(), all_rate_types()):
        back = mechanism_from_dict(mechanism_to_dict(m))
        np.testing.assert_array_equal(CompiledMechanism(back).species_columns, CompiledMechanism(m).species_columns)
        for key, a in m.flat().items():
            np.testing.assert_array_equal(np.asarray(back.flat()[key]), np.asarray(a), err_msg=key)
        assert back.custom_param_labels() == m.custom_param_labels()
        np.testing.assert_array_equal(back.atol(), m.atol())
