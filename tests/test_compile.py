"""Symbolic compile (host, no GPU) against micm's own builder."""
import numpy as np
import pytest

import oracle
from micm_b200.solver import CompiledMechanism
from micm_b200 import synthetic

from mechanisms import mechanism_set

pytestmark = pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")

MECHS = mechanism_set()


@pytest.mark.parametrize("name", sorted(MECHS))
def test_numbering_matches_reference(name):
    m = MECHS[name]
    cm = CompiledMechanism(m)
    ref = oracle.Reference(m, tableau=3)
    np.testing.assert_array_equal(cm.species_columns, ref.species_columns)
    np.testing.assert_array_equal(cm.reaction_columns, ref.reaction_columns)
    np.testing.assert_array_equal(cm.param_columns, ref.param_columns)
    np.testing.assert_array_equal(cm.rows, ref.rows)
    np.testing.assert_array_equal(cm.cols, ref.cols)
    assert cm.info["n_custom_params"] == ref.n_params


def test_numbering_without_reorder():
    m = synthetic.synthetic_mechanism(60, 120, seed=601)
    m.reorder_state = False
    cm = CompiledMechanism(m)
    ref = oracle.Reference(m, tableau=3)
    np.testing.assert_array_equal(cm.species_columns, np.arange(60))
    np.testing.assert_array_equal(cm.species_columns, ref.species_columns)
    np.testing.assert_array_equal(cm.rows, ref.rows)
    np.testing.assert_array_equal(cm.cols, ref.cols)


def test_large_mechanism_numbering():
    # a denser hub structure than the default, so the LU fill outgrows shared memory
    m = synthetic.synthetic_mechanism(600, 1500, seed=6001, hub_fraction=0.07, window=12, hub_skew=1.0)
    cm = CompiledMechanism(m)
    ref = oracle.Reference(m, tableau=4)
    np.testing.assert_array_equal(cm.species_columns, ref.species_columns)
    np.testing.assert_array_equal(cm.rows, ref.rows)
    np.testing.assert_array_equal(cm.cols, ref.cols)
    assert cm.info["jacobian_nnz"] == ref.nnz > 16384  # LU fill beyond one shared-memory working set


def test_schedules_are_consistent():
    """Every LU item's dependencies lie in earlier levels (checked on the host
    from the patterns: Crout update count equals micm's Mozart op count)."""
    m = synthetic.synthetic_mechanism(210, 440, seed=2101)
    cm = CompiledMechanism(m)
    rows, cols = cm.rows, cm.cols
    S = m.n_species
    nz = set(zip(rows.tolist(), cols.tolist()))
    # Mozart op count: sum over pivots of |L col| * |U row|
    updates = 0
    for i in range(S):
        nl = sum(1 for j in range(i + 1, S) if (j, i) in nz)
        nu = sum(1 for k in range(i + 1, S) if (i, k) in nz)
        updates += nl * nu
    assert cm.info["lu_updates"] == updates
    assert cm.info["lu_lower"] == sum(1 for r, c in nz if r > c)


def test_invalid_mechanism_rejected():
    from micm_b200._native import MicmbError
    m = synthetic.readme_mechanism()
    m.reactions[0].reactants = [7]
    with pytest.raises(MicmbError):
        CompiledMechanism(m)


def test_register_blocked_schedules_are_kept_for_the_benchmark_mechanisms():
    """The compiler keeps the register-blocked LU and solves only when they
    reproduce the serial schedules bit for bit on random values (a host check
    at build time); every benchmark mechanism passes it."""
    from micm_b200 import micm_bench, synthetic
    from micm_b200.solver import CompiledMechanism
    mechs = [synthetic.CONFIGS[n]["mech"]() for n in ("readme", "c210", "c60_adjoint", "c600")]
    mechs += [micm_bench.mechanism(n) for n in ("ts1", "chapman")]
    for m in mechs:
        info = CompiledMechanism(m).info
        assert info["blocked_schedules"] == 1
        assert info["lu_blocked_ops"] <= info["lu_updates"]
