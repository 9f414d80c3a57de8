"""micm's TS1 benchmark mechanism (MOZART-TS1: 209 state species, 547
reactions -- Arrhenius, Troe, user-defined photolysis and surface reactions
with a third body M) and the initial state of micm's own benchmark
(test/benchmark/ts1_mechanism.hpp, bench::Ts1::InitState; driven by
test/benchmark/micm_bench.cpp with ThreeStageRosenbrockParameters, dt = 30 s).

The mechanism and initial state are read from tests/golden/ts1_mechanism.json,
which tests/golden/make_ts1.py writes from micm itself (micm builds the
mechanism from its header and the program prints it in this repository's
JSON description; see micm_b200.mechanism.mechanism_from_dict).
"""
from __future__ import annotations

import json
import os
from typing import Dict, Optional

import numpy as np

from .mechanism import Mechanism, ideal_air_density, mechanism_from_dict

FIXTURE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                       "ts1_mechanism.json")
TABLEAU = 3          # micm_bench: RosenbrockSolverParameters::ThreeStageRosenbrockParameters()
DT = 30.0            # micm_bench's default time step [s]


def _document(path: Optional[str] = None) -> dict:
    with open(path or FIXTURE) as f:
        return json.load(f)


def mechanism(path: Optional[str] = None, absolute_tolerance: Optional[float] = None) -> Mechanism:
    """TS1 as micm builds it.  The absolute tolerance is micm's builder default
    (1e-3, what micm_bench runs with) unless one is given for every species."""
    m = mechanism_from_dict(_document(path))
    if absolute_tolerance is not None:
        m.absolute_tolerance = np.full(m.n_species, float(absolute_tolerance))
    return m


def inputs(n_cells: int, seed: Optional[int] = None, path: Optional[str] = None) -> Dict[str, np.ndarray]:
    """micm_bench's initial state on every cell (T = 287.45 K, P = 101319.9 Pa,
    the benchmark's concentrations and photolysis / aerosol parameters).  With
    a seed, each cell is varied: concentrations scaled by 10**U(-0.5, 0.5),
    T shifted by U(-30, 10) K and photolysis rates scaled by U(0, 1)."""
    doc = _document(path)
    mech = mechanism_from_dict(doc)
    init = doc["init"]
    y = np.array([init["concentrations"][s] for s in mech.species], dtype=np.float64)
    labels = mech.custom_param_labels()
    p = np.array([init["custom_parameters"][l] for l in labels], dtype=np.float64)
    n = int(n_cells)
    T = np.full(n, float(init["temperature"]))
    P = np.full(n, float(init["pressure"]))
    conc = np.tile(y, (n, 1))
    params = np.tile(p, (n, 1))
    if seed is not None:
        rng = np.random.default_rng(seed)
        conc *= 10.0 ** rng.uniform(-0.5, 0.5, size=conc.shape)
        T += rng.uniform(-30.0, 10.0, size=n)
        photolysis = np.array([l.startswith("j") for l in labels])
        params[:, photolysis] *= rng.uniform(0.0, 1.0, size=(n, int(photolysis.sum())))
    return dict(temperature=T, pressure=P, air_density=ideal_air_density(P, T), concentrations=conc,
                custom_params=params)


def micm_columns(path: Optional[str] = None) -> Dict[str, Dict[str, int]]:
    """micm's own state columns for every species and custom parameter."""
    return _document(path)["micm_columns"]
